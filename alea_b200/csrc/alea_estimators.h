// Device observable estimators (alea_estimators.cu) as the C ABI calls them;
// not part of include/alea_gpu.h.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/alea_gpu.h"
#include "alea_dev.cuh"

namespace alea_gpu {

struct EstimatorSet;

// Every call returns ALEA_OK or an ALEA_ERR_* code with a message in err.
// Device memory is allocated and freed stream-ordered on `st`.
int est_add(EstimatorSet*& set, const DevSys& s, const alea_gpu_estimator_spec& spec, cudaStream_t st,
            std::string& err, int* id);
void est_free(EstimatorSet*& set, cudaStream_t st);
int est_count(const EstimatorSet* set);
int est_reset(EstimatorSet* set, cudaStream_t st, std::string& err);
int est_start_block(EstimatorSet* set, cudaStream_t st, std::string& err);
// Where a measurement's configurations are: walker records (stride s.rec,
// positions at s.o_pos, weight at s.o_scal + S_WEIGHT) or compact position
// rows (stride np * 2, offset 0, no weight); configuration c of the
// measurement is block idx[c] (idx null: block c).
struct EstSource {
    const double* base;
    long stride;
    int o_pos;
    int o_w;              // -1: the blocks hold no weight
    const int* idx;       // device [n] or null
    int n;                // configurations measured
};

// One measurement of every estimator of the set.  d_weights: device [n] or
// null (the blocks' own weights); unit: every weight 1.  Adds the launches to
// *launches.
int est_accumulate(EstimatorSet* set, const DevSys& s, const EstSource& src, const double* d_weights, bool unit,
                   int chains, const int2* pairs, int npair, cudaStream_t st, std::string& err, uint64_t* launches);
// Reads the running blocks back (adds the bytes to *d2h), stores the block
// estimates, zeroes the running blocks.
int est_stop_block(EstimatorSet* set, cudaStream_t st, std::string& err, uint64_t* d2h);
int est_info(const EstimatorSet* set, int id, alea_gpu_estimator_desc* out);
int est_blocks(const EstimatorSet* set, int id, double* out);
int est_kvectors(const EstimatorSet* set, int id, int* n1, int* n2, double* kx, double* ky, int* shell_of,
                 double* shell_k, int* shell_count);

}  // namespace alea_gpu
