// Internal hooks between the C ABI (alea_capi.cu) and the server
// (alea_serve.cpp); not part of include/alea_gpu.h.
#pragma once

#include <atomic>
#include <cstddef>

#include "../../include/alea_gpu.h"

namespace alea_gpu {

// The run loops of `c` (alea_gpu_vmc_run / alea_gpu_dmc_run) return
// ALEA_ERR_CANCELLED at their next step once *flag is nonzero.
void set_cancel_flag(alea_gpu_ctx* c, const std::atomic<int>* flag);

// Device bytes of a context of `capacity` walkers of `sys` running
// `n_substeps` sweeps per step (the server's admission estimate).
size_t footprint_bytes(const alea_gpu_system* sys, int capacity, int n_substeps);

}  // namespace alea_gpu
