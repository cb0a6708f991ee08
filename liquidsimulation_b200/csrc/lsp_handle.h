// The opaque lsp_solver handle of the C ABI and the error channel shared by the
// translation units that implement entry points.
#pragma once

#include <new>
#include <string>

#include "engine.h"

struct lsp_solver {
    lsp::Engine* e;
};

namespace lsp {
// Sets the message lsp_last_error() returns on this thread.
void set_last_error(const std::string& message);

// Device address of lsp_mlp_gradient_static's fixed scratch array on `device`, which must be
// the current device (looked up once per device; mlp_static.cu).
float* scratch_on(int device);

// Runs an entry point's body: LSP_OK, or the status code of the error it threw with the
// message kept for lsp_last_error() (host allocation failures map to LSP_ERR_CAPACITY).
template <typename F>
int guard(F&& f)
{
    try {
        f();
        return LSP_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return LSP_ERR_CAPACITY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return LSP_ERR_INVALID;
    }
}
}  // namespace lsp
