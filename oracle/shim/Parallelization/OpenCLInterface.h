// Test-infrastructure shim, not product code.
//
// Stands in for the reference's OpenCL backend header
// (LiquidPhysics/include/Parallelization/OpenCLInterface.h:1-63) so that the
// reference's sequential CPU solver can be compiled here, where no OpenCL headers
// or runtime exist. The backend reports itself invalid, which makes
// SPHSolver::SPHSolver (LiquidPhysics/src/SPHSolver.cpp:71-85) select
// ParallelizationType::NONE, the sequential CPU path. Every other method is a
// no-op and is never reached on that path.
//
// This directory must come before LiquidPhysics/include on the include path.
#pragma once

#include "Parallelization/ParallelComputationInterface.h"

namespace LiPhEn {
	class OpenCLInterface : public ParallelComputationInterface
	{
	public:
		OpenCLInterface() {}

		virtual void initialize(bool) { m_isValid = false; m_hasCPU = false; m_hasGPU = false; }
		virtual void reinitContext(ParallelSources, ParallelDeviceType, bool) {}
		virtual ParallelKernel* createKernel(const char*) { return nullptr; }
		virtual ParallelBuffer* createBuffer(ParallelBufferType, unsigned int) { return nullptr; }
		virtual void executeKernel(ParallelKernel*, unsigned int, unsigned int = 0) {}
		virtual void writeToBuffer(ParallelBuffer*, void*, unsigned int, bool) {}
		virtual void readFromBuffer(ParallelBuffer*, void*, unsigned int, bool) {}
		virtual void fillBuffer(ParallelBuffer*, int, unsigned int) {}
		virtual void waitUntilFinished() {}
	};
}
