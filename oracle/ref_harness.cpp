// Test-infrastructure harness, not product code.
//
// A C entry-point layer over the UNMODIFIED reference sequential CPU solver
// (LiquidPhysics/src/*.cpp, compiled where it lies by oracle/Makefile with the
// OpenCL shim in oracle/shim). Python loads the resulting oracle/_ref/libref_sph.so
// with ctypes to (a) pin the project's own CPU restatement (oracle/sph_oracle.cpp)
// bit for bit, (b) generate golden fixtures, and (c) time the reference's CPU path
// as the baseline. Nothing in the product links or loads this library.
//
// Observation hooks (none of them change the reference's arithmetic):
//  * Harness<Base> derives from SPHSolver / PCISPHSolver to read protected state:
//    the particle mass (SPHSolver.h:132), the kernel lookup tables (SPHSolver.h:124-126)
//    and the start-of-step neighbour lists (SPHSolver.h:123), captured in an
//    override of onEndUpdate (SPHSolver.cpp:384-397) before the base class clears them.
//  * CountingCollider is a StaticCollisionObject that never reports a collision but
//    counts detectCollisionWithParticle calls. SPHSolver::handleCollision
//    (SPHSolver.cpp:370-382) calls it once per particle per collision pass, so for
//    PCISPH the number of predict-correct iterations of the last step is
//    calls / N - 1 (PCISPHSolver.cpp:84-97 once per iteration, plus the final
//    SPHSolver::handleCollisions at SPHSolver.cpp:337-355).
#include "SPHSolver.h"
#include "PCISPHSolver.h"
#include "Particles/PCISPHParticle.h"
#include "Collision/StaticCollisionBox.h"
#include "Collision/StaticCollisionSphere.h"

#include <cstring>
#include <unordered_map>
#include <vector>

using namespace LiPhEn;

namespace {

class CountingCollider : public StaticCollisionObject
{
public:
	CountingCollider() : StaticCollisionObject(Vector3D(0.f, 0.f, 0.f)) {}
	mutable long long calls = 0;

protected:
	virtual StaticCollisionInfo detectCollisionWithParticle(ParticleCollisionData particleData) const
	{
		calls++;
		StaticCollisionInfo info;
		info.collisionNormal = Vector3D(0.f, 0.f, 0.f);
		info.collisionPoint = particleData.position;
		info.foundCollision = false;
		return info;
	}
};

struct RefHandle;

template <class Base>
class Harness : public Base
{
public:
	RefHandle* owner = nullptr;
	bool capture = false;
	std::vector<int> nbrOffsets;   // CSR offsets, size N+1
	std::vector<int> nbrIndex;     // neighbour indices in caller order

	void forceMass(float m) { this->m_particleMass = m; }
	float mass() const { return this->m_particleMass; }
	float kernelRadius() const { return this->m_kernelRadius; }
	std::vector<SPHParticle*>& particles() { return this->m_particles; }
	void tables(float* out)
	{
		std::vector<float> t[5] = {
			this->m_defaultKernel.getKernelWeights(),
			this->m_defaultKernel.getFirstDerivativeWeights(),
			this->m_defaultKernel.getSecondDerivativeWeights(),
			this->m_pressureKernel.getFirstDerivativeWeights(),
			this->m_viscosityKernel.getSecondDerivativeWeights(),
		};
		size_t n = t[0].size();
		for (int k = 0; k < 5; k++)
			std::memcpy(out + k * n, t[k].data(), n * sizeof(float));
	}
	float divisionStep() { return this->m_defaultKernel.getDivisionStep(); }

protected:
	virtual void onEndUpdate();
};

struct RefHandle
{
	bool pcisph = false;
	Harness<SPHSolver>* sph = nullptr;
	Harness<PCISPHSolver>* pci = nullptr;
	CountingCollider* counter = nullptr;  // owned by the solver once added
	std::unordered_map<SPHParticle*, int> index;
	long long countBefore = 0;
	int lastIterations = -1;

	SPHSolver* solver() { return pcisph ? static_cast<SPHSolver*>(pci) : static_cast<SPHSolver*>(sph); }
	std::vector<SPHParticle*>& particles() { return pcisph ? pci->particles() : sph->particles(); }
};

template <class Base>
void Harness<Base>::onEndUpdate()
{
	if (capture && owner)
	{
		const auto& lists = this->m_cachedNeighborLists;
		nbrOffsets.assign(lists.size() + 1, 0);
		nbrIndex.clear();
		for (size_t i = 0; i < lists.size(); i++)
		{
			for (SPHParticle* p : lists[i])
				nbrIndex.push_back(owner->index[p]);
			nbrOffsets[i + 1] = (int)nbrIndex.size();
		}
	}
	Base::onEndUpdate();
}

}  // namespace

extern "C" {

void* ref_create(int pcisph)
{
	RefHandle* h = new RefHandle();
	h->pcisph = pcisph != 0;
	if (h->pcisph) { h->pci = new Harness<PCISPHSolver>(); h->pci->owner = h; }
	else { h->sph = new Harness<SPHSolver>(); h->sph->owner = h; }
	return h;
}

void ref_destroy(void* p)
{
	RefHandle* h = (RefHandle*)p;
	if (h->pcisph) delete h->pci; else delete h->sph;
	delete h;
}

int ref_parallelization_type(void* p)
{
	return (int)((RefHandle*)p)->solver()->getParallelizationType();
}

// Parameter setters, in the reference's own units (SPHSolver.h:57-69, PCISPHSolver.h:19-20).
void ref_set_gravity(void* p, float x, float y, float z) { ((RefHandle*)p)->solver()->setGravity(Vector3D(x, y, z)); }
void ref_set_particle_radius(void* p, float v) { ((RefHandle*)p)->solver()->setParticleRadius(v); }
void ref_set_kernel_radius_factor(void* p, float v) { ((RefHandle*)p)->solver()->setKernelRadiusFactor(v); }
void ref_set_rest_density(void* p, float v) { ((RefHandle*)p)->solver()->setRestDensity(v); }
void ref_set_viscosity(void* p, float v) { ((RefHandle*)p)->solver()->setViscosityCoefficient(v); }
void ref_set_stiffness(void* p, float v) { ((RefHandle*)p)->solver()->setPressureStiffnessCoefficient(v); }
void ref_set_negative_pressure_factor(void* p, float v) { ((RefHandle*)p)->solver()->setNegativePressureFactor(v); }
void ref_set_surface_tension(void* p, float v) { ((RefHandle*)p)->solver()->setSurfaceTensionCoefficient(v); }
void ref_set_surface_tension_threshold(void* p, float v) { ((RefHandle*)p)->solver()->setSurfaceTensionThreshold(v); }
void ref_set_restitution(void* p, float v) { ((RefHandle*)p)->solver()->setRestitutionCoefficient(v); }
void ref_set_friction(void* p, float v) { ((RefHandle*)p)->solver()->setFrictionCoefficient(v); }
void ref_set_pci_iterations(void* p, int v) { RefHandle* h = (RefHandle*)p; if (h->pcisph) h->pci->setMinIterations(v); }
void ref_set_pci_eta(void* p, float v) { RefHandle* h = (RefHandle*)p; if (h->pcisph) h->pci->setMaxDensityErrorRatio(v); }
void ref_force_mass(void* p, float m)
{
	RefHandle* h = (RefHandle*)p;
	if (h->pcisph) h->pci->forceMass(m); else h->sph->forceMass(m);
}
void ref_capture_neighbors(void* p, int on)
{
	RefHandle* h = (RefHandle*)p;
	if (h->pcisph) h->pci->capture = on != 0; else h->sph->capture = on != 0;
}

float ref_mass(void* p) { RefHandle* h = (RefHandle*)p; return h->pcisph ? h->pci->mass() : h->sph->mass(); }
float ref_kernel_radius(void* p) { RefHandle* h = (RefHandle*)p; return h->pcisph ? h->pci->kernelRadius() : h->sph->kernelRadius(); }
float ref_division_step(void* p) { RefHandle* h = (RefHandle*)p; return h->pcisph ? h->pci->divisionStep() : h->sph->divisionStep(); }

// out: 5 x 1001 floats: poly6 W, poly6 dW, poly6 d2W, spiky dW, viscosity d2W.
void ref_tables(void* p, float* out)
{
	RefHandle* h = (RefHandle*)p;
	if (h->pcisph) h->pci->tables(out); else h->sph->tables(out);
}

// Adds n particles (positions xyz[3n], velocities vel[3n] or NULL).
void ref_add_particles(void* p, const float* xyz, const float* vel, int n)
{
	RefHandle* h = (RefHandle*)p;
	for (int i = 0; i < n; i++)
	{
		SPHParticle* q = h->pcisph ? new PCISPHParticle() : new SPHParticle();
		q->setPosition(Vector3D(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
		if (vel) q->setVelocity(Vector3D(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]));
		int idx = (int)h->particles().size();
		h->index[q] = idx;
		h->solver()->addParticle(q);
	}
}

void ref_add_box(void* p, const float* center, const float* half, int boundary)
{
	((RefHandle*)p)->solver()->addStaticCollisionObject(new StaticCollisionBox(
		Vector3D(center[0], center[1], center[2]), Vector3D(half[0], half[1], half[2]),
		boundary ? StaticCollisionObjectType::BOUNDARY : StaticCollisionObjectType::OBSTACLE));
}

void ref_add_sphere(void* p, const float* center, float radius, int boundary)
{
	((RefHandle*)p)->solver()->addStaticCollisionObject(new StaticCollisionSphere(
		Vector3D(center[0], center[1], center[2]), radius,
		boundary ? StaticCollisionObjectType::BOUNDARY : StaticCollisionObjectType::OBSTACLE));
}

// Adds the iteration-counting collider. Call after the real colliders; it never collides,
// so its place in the list does not change results.
void ref_add_iteration_counter(void* p)
{
	RefHandle* h = (RefHandle*)p;
	if (!h->counter)
	{
		h->counter = new CountingCollider();
		h->solver()->addStaticCollisionObject(h->counter);
	}
}

int ref_count(void* p) { return (int)((RefHandle*)p)->particles().size(); }

void ref_step(void* p, float dt)
{
	RefHandle* h = (RefHandle*)p;
	long long before = h->counter ? h->counter->calls : 0;
	h->solver()->update(dt);
	if (h->counter)
	{
		long long n = (long long)h->particles().size();
		long long calls = h->counter->calls - before;
		h->lastIterations = n > 0 ? (int)(calls / n - 1) : 0;
	}
}

void ref_steps(void* p, float dt, int steps)
{
	for (int s = 0; s < steps; s++) ref_step(p, dt);
}

int ref_last_iterations(void* p) { return ((RefHandle*)p)->lastIterations; }

// Field ids for ref_get / ref_set.
enum {
	F_POS = 0, F_VEL = 1, F_HALF = 2, F_DENSITY = 3, F_PRESSURE = 4, F_FIRST = 5,
	F_PRED_DENSITY = 6, F_DENSITY_ERROR = 7, F_PRED_POS = 8, F_PRED_HALF = 9, F_PRED_PFORCE = 10,
};

static void put3(float* out, int i, const Vector3D& v) { out[3 * i] = v.getX(); out[3 * i + 1] = v.getY(); out[3 * i + 2] = v.getZ(); }

int ref_get(void* p, int field, float* out)
{
	RefHandle* h = (RefHandle*)p;
	std::vector<SPHParticle*>& ps = h->particles();
	for (int i = 0; i < (int)ps.size(); i++)
	{
		SPHParticle* q = ps[i];
		PCISPHParticle* c = h->pcisph ? static_cast<PCISPHParticle*>(q) : nullptr;
		switch (field)
		{
		case F_POS: put3(out, i, q->getPosition()); break;
		case F_VEL: put3(out, i, q->getVelocity()); break;
		case F_HALF: put3(out, i, q->getHalfVelocity()); break;
		case F_DENSITY: out[i] = q->getDensity(); break;
		case F_PRESSURE: out[i] = q->getPressure(); break;
		case F_FIRST: out[i] = q->getIsFirstTimeStep() ? 1.f : 0.f; break;
		case F_PRED_DENSITY: if (!c) return -1; out[i] = c->getPredictedDensity(); break;
		case F_DENSITY_ERROR: if (!c) return -1; out[i] = c->getDensityError(); break;
		case F_PRED_POS: if (!c) return -1; put3(out, i, c->getPredictedPosition()); break;
		case F_PRED_HALF: if (!c) return -1; put3(out, i, c->getPredictedHalfVelocity()); break;
		case F_PRED_PFORCE: if (!c) return -1; put3(out, i, c->getPredictedPressureForce()); break;
		default: return -1;
		}
	}
	return 0;
}

// Injects the persistent per-particle state: x, v, v_half, v_half_old (xyz each) and the
// first-step flag. The reference keeps exactly these across steps; forces are cleared by
// SPHParticle::integrate (SPHParticle.cpp:43) and density/pressure are recomputed.
void ref_set_state(void* p, const float* x, const float* v, const float* half, const float* oldHalf, const int* first)
{
	RefHandle* h = (RefHandle*)p;
	std::vector<SPHParticle*>& ps = h->particles();
	for (int i = 0; i < (int)ps.size(); i++)
	{
		SPHParticle* q = ps[i];
		q->setPosition(Vector3D(x[3 * i], x[3 * i + 1], x[3 * i + 2]));
		q->setVelocity(Vector3D(v[3 * i], v[3 * i + 1], v[3 * i + 2]));
		q->setHalfVelocity(Vector3D(half[3 * i], half[3 * i + 1], half[3 * i + 2]));
		q->setOldHalfVelocity(Vector3D(oldHalf[3 * i], oldHalf[3 * i + 1], oldHalf[3 * i + 2]));
		q->setIsFirstTimeStep(first[i] != 0);
	}
}

// Neighbour lists captured at the end of the last step (after ref_capture_neighbors(h, 1)).
int ref_neighbor_total(void* p)
{
	RefHandle* h = (RefHandle*)p;
	return (int)(h->pcisph ? h->pci->nbrIndex.size() : h->sph->nbrIndex.size());
}

void ref_neighbor_lists(void* p, int* offsets, int* index)
{
	RefHandle* h = (RefHandle*)p;
	std::vector<int>& o = h->pcisph ? h->pci->nbrOffsets : h->sph->nbrOffsets;
	std::vector<int>& x = h->pcisph ? h->pci->nbrIndex : h->sph->nbrIndex;
	std::memcpy(offsets, o.data(), o.size() * sizeof(int));
	std::memcpy(index, x.data(), x.size() * sizeof(int));
}

}  // extern "C"
