// Context management of the drop-in shims (hpc_shim.cpp, hpc_shim_loop.cpp).
#pragma once

#include "stack_and_level.h"
#include "hpcrack.h"

// Device context of a hierarchy (created from the Stack's geometry on first use).
hpc_ctx* hpc_shim_context(Stack* U);
// Destroys every context the shims created.
void hpc_shim_release_all();
