// Kernel entry points shared by alea_kernels.cu and the host code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "alea_dev.cuh"

namespace alea_gpu {

struct SweepParams {
    int mode;                 // 0 VMC step, 1 DMC advance
    int n_sub;                // sweeps per call
    int drift;                // VMC: Langevin proposals
    double tau;
    const double* sigma;      // [np*dim] sqrt(tau / m)
    double etrial, eref, e_cut, e_max;
};

// Walker kernels, one CTA of nt threads (32, 64 or 128) per walker and nw
// CTAs; host-side launchers that dispatch on nt.
cudaError_t reserve_smem(size_t smem);
cudaError_t launch_evaluate(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                            double* records, const int2* pairs, int npair);
// d ln psi / d p of the nopt optimisable parameters for nw walkers, out [nopt][nw].
cudaError_t launch_param_derivatives(int nw, cudaStream_t st, const DevSys& s, const double* records,
                                     const DevOpt* opts, int nopt, double* out);
// The Gaussian-width parameters (kind 1) of the same list: out [nopt][nw] and,
// when dgrad/dlap are given, their rows of the curvature planes; scratch holds
// 3 maxN^2 doubles per CTA of the grid.
cudaError_t launch_orbital_param_derivatives(int nw, int grid, cudaStream_t st, const DevSys& s,
                                            const double* records, const DevOpt* opts, int nopt, double* out,
                                            double* dgrad, double* dlap, double* scratch);
// d(grad ln psi)/dp and d(lap ln psi)/dp of the nopt parameters, [nopt][np*2][nw]
// each; entries of particles outside a parameter's term are left as they are.
cudaError_t launch_param_grad_derivatives(int nw, cudaStream_t st, const DevSys& s, const double* records,
                                          const DevOpt* opts, int nopt, double* dgrad, double* dlap);
// The backflow channels' parameters' curvature terms (one CTA per walker)
// and the dynamic shared memory that kernel takes.
size_t bf_curvature_smem(const DevSys& s);
cudaError_t launch_bf_curvature(int nw, cudaStream_t st, const DevSys& s, const double* records, const DevOpt* opts,
                                int nopt, double* dgrad, double* dlap);
// Measured FP64 FMA throughput of `device` in TFLOP/s (a register-only loop).
cudaError_t measure_fp64_peak(int device, double* tflops);
// Potential energy of n stored configurations rows[idx[c]] into out[c].
cudaError_t launch_potential(int nt, int n, size_t smem, cudaStream_t st, const DevSys& s, const double* rows,
                             const int* idx, const int2* pairs, int npair, double* out);
cudaError_t launch_measure(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                           double* records, const int2* pairs, int npair);
cudaError_t launch_move(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                        double* records, int p, const double* new_pos, const uint8_t* accept,
                        double* out);
cudaError_t launch_sweep(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                         double* records, const double* randoms, long stride,
                         const SweepParams& prm, const int2* pairs, int npair);
// The one-warp sweep (alea_fast.cu): systems of real determinants and
// group-wise pair terms with at most 64 particles, 64 orbitals per block and
// 64 image-sum k-vectors.  launch_sweep takes it for 32-thread walkers unless
// ALEA_GPU_SWEEP=generic is set in the environment.
bool fast_sweep_eligible(const DevSys& s);
cudaError_t reserve_smem_fast(size_t smem);
cudaError_t launch_sweep_fast(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records,
                              const double* randoms, long stride, const SweepParams& prm, const int2* pairs,
                              int npair);
// One context's share of a packed sweep launch: its walkers are
// [first, first + nw) of the launch's global walker index, swept with its own
// system (a device copy of its DevSys), records, random numbers and
// parameters.  Jobs are in increasing `first`.
struct BatchJob {
    const DevSys* sys;
    double* records;
    const double* randoms;
    long stride;
    SweepParams prm;
    const int2* pairs;
    int npair;
    int first, nw;
};
// Packed sweeps of n_jobs jobs, `total` walkers in all, one 32-thread CTA per
// walker at a time: the one-warp body (alea_fast.cu, every job fast-sweep
// eligible; zero_energy: some job has a zero-energy term; complex_det: every
// job's determinants are complex, none otherwise) or the generic body
// with nt threads per walker (alea_kernels.cu, any system; each job packed
// with the contexts of its own thread count).  grid >= total: one CTA per
// walker; grid < total: persistent CTAs take walkers from the counter *next
// (zero before the launch).  The walker's arithmetic is that of launch_sweep
// on its own context whatever the grid.  reserve_smem covers both kernels.
cudaError_t launch_sweep_fast_batch(bool zero_energy, bool complex_det, const BatchJob* jobs, int n_jobs, int total,
                                    int grid, size_t smem, int* next, cudaStream_t st);
cudaError_t launch_sweep_generic_batch(int nt, const BatchJob* jobs, int n_jobs, int total, int grid, size_t smem,
                                       int* next, cudaStream_t st);
// Resident CTAs per SM of the generic packed kernel of nt threads at `smem`.
int batch_ctas_per_sm(int nt, size_t smem);
// Resident CTAs per SM of the packed one-warp kernel (real or complex form).
int fast_batch_ctas_per_sm(bool complex_det, size_t smem);
// The one-warp Jastrow-only sweep (alea_boson.cu): no determinant, no image
// sum, group-wise pair terms, 65 to 256 particles, in the one-warp layout.
// launch_sweep takes it for any thread count unless ALEA_GPU_SWEEP=generic.
bool boson_sweep_eligible(const DevSys& s);
cudaError_t reserve_smem_boson(size_t smem);
cudaError_t launch_sweep_boson(int nw, cudaStream_t st, const DevSys& s, double* records, const double* randoms,
                               long stride, const SweepParams& prm, const int2* pairs, int npair);
cudaError_t launch_sweep_boson_batch(bool zero_energy, const BatchJob* jobs, int n_jobs, int total, int grid,
                                     size_t smem, int* next, cudaStream_t st);
int boson_batch_ctas_per_sm(size_t smem);
// The walker of global index w of a packed launch: its job by binary search
// over the jobs' first indices.
__device__ __forceinline__ int batch_job_of(const BatchJob* jobs, int n_jobs, int w) {
    int lo = 0, hi = n_jobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].first <= w) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Next walker of a packed launch for this CTA: blockIdx.x once (grid >= total)
// or from the shared counter; -1 when none is left.
__device__ __forceinline__ int batch_next(int total, int* next, int* slot, bool first_round) {
    if (gridDim.x >= total) return first_round && static_cast<int>(blockIdx.x) < total ? static_cast<int>(blockIdx.x) : -1;
    __syncthreads();
    if (threadIdx.x == 0) *slot = atomicAdd(next, 1);
    __syncthreads();
    const int w = *slot;
    return w < total ? w : -1;
}

// The FP32 form of the one-warp sweep (alea_fast32.cu), for the one-warp
// sweep's systems without zero-energy terms; launch_sweep takes it whenever
// DevSys::f32 is set.
bool f32_sweep_eligible(const DevSys& s);
cudaError_t reserve_smem_f32(size_t smem);
cudaError_t launch_sweep_f32(int nw, cudaStream_t st, const DevSys& s, double* records, const double* randoms,
                             long stride, const SweepParams& prm, const int2* pairs, int npair);
// One thread per random stream: its crowd's randoms of n_sweeps sweeps, per
// particle `dim` Gaussians then one uniform, [(sweep·np + p)·(dim+1)·stride +
// d·stride + w] (src/qmc/sweep_blocking.h:39-48).
__global__ void draw_kernel(uint64_t* states, int n_streams, int nw, int np, long stride,
                            int n_sweeps, const uint64_t* zk, const double* zw, const double* zf,
                            double zr, double* out, int dim);
// The three-dimensional walker kernels (alea_bf3d.cu): evaluation and the
// VMC/DMC sweep, one CTA of 128 threads per walker, smem bytes each.
cudaError_t launch_evaluate3(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records);
cudaError_t launch_sweep3(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records,
                          const double* randoms, long stride, const SweepParams& prm);
__global__ void gather_kernel(double* dst, const double* src, const int* src_idx, int n, long rec);
__global__ void scalar_kernel(const double* records, int nw, long rec, int offset, double* out);
__global__ void to_soa_kernel(const double* records, int nw, long rec, int offset, int n, double* out);
__global__ void from_soa_kernel(double* records, int nw, long rec, int offset, int n, const double* in);
__global__ void set_scalar_kernel(double* records, int nw, long rec, int offset, double value);
// AoS rows [w][i] of the n doubles at `offset` of each record; the inverse
// takes row w mod n_rows for walker w.
__global__ void to_rows_kernel(const double* records, int nw, long rec, int offset, int n, double* out);
__global__ void from_rows_kernel(double* records, int nw, long rec, int offset, int n, const double* rows,
                                 int n_rows);
// idx[w] = w mod n_src
__global__ void cycle_index_kernel(int* idx, int nw, int n_src);

}  // namespace alea_gpu
