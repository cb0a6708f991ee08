// The opaque lsp_solver handle of the C ABI and the error channel shared by the
// translation units that implement entry points.
#pragma once

#include <string>

#include "engine.h"

struct lsp_solver {
    lsp::Engine* e;
};

namespace lsp {
// Sets the message lsp_last_error() returns on this thread.
void set_last_error(const std::string& message);
}  // namespace lsp
