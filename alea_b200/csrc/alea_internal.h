// Internal hooks between the C ABI (alea_capi.cu) and the server
// (alea_serve.cpp); not part of include/alea_gpu.h.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/alea_gpu.h"

struct alea_gpu_packed;

namespace alea_gpu {

// The run loops of `c` (alea_gpu_vmc_run / alea_gpu_dmc_run) return
// ALEA_ERR_CANCELLED at their next step once *flag is nonzero.
void set_cancel_flag(alea_gpu_ctx* c, const std::atomic<int>* flag);

// Device bytes of a context of `capacity` walkers of `sys` running
// `n_substeps` sweeps per step (the server's admission estimate).
size_t footprint_bytes(const alea_gpu_system* sys, int capacity, int n_substeps);

// Packed VMC runs (alea_capi.cu, "packed VMC runs"): several contexts'
// runs stepped together, one sweep launch per sweep body per step.
int packed_create(int device, alea_gpu_packed** out);
void packed_destroy(alea_gpu_packed* P);
const std::string& packed_error(const alea_gpu_packed* P);
// Body classes of the packed sweeps and the class of a context's walkers
// (0 one-warp real, 1-3 generic of 32, 64, 128 threads, 4 one-warp complex,
// 5 one-warp Jastrow-only).
constexpr int kPackedClasses = 6;
int packed_class(const alea_gpu_ctx* c);
// Join with a context whose walkers are uploaded; *slot numbers the run.
int packed_add(alea_gpu_packed* P, alea_gpu_ctx* c, const alea_gpu_run_config& cfg, int* slot);
int packed_active(const alea_gpu_packed* P);
// One step of every run still going.
int packed_step(alea_gpu_packed* P);
// Whether run `slot` has finished, with its status and result.
bool packed_done(const alea_gpu_packed* P, int slot, int* status, alea_gpu_run_result* res);
// Stop run `slot` before its next step (status ALEA_ERR_CANCELLED).
void packed_cancel(alea_gpu_packed* P, int slot);
// Forget the finished runs; the slots of the others renumber in order.
void packed_prune(alea_gpu_packed* P);
uint64_t packed_launches(const alea_gpu_packed* P);

}  // namespace alea_gpu
