// Observable estimators on the device: pair correlation g(r)
// (src/estimators/pair_correlation.cpp), the density grid
// (src/estimators/density.cpp) and the structure factor S(k) with ρ_g(k)
// (src/estimators/structure_factor.cpp).
//
// A measurement reads each walker's positions from its record in HBM; one
// warp per CTA owns one row of running sums (in shared memory when it fits,
// else in its own slice of an HBM scratch) and bins a contiguous range of
// walkers into it.  Within a walker the lanes take 32 pairs (particles,
// k-vectors) at a time; lanes that land in the same bin are counted with
// match.any and their leader adds weight × count, so no two lanes of a warp
// ever add to one address and a row's sums have a fixed order.  Two more
// kernels add a chain's rows into its running block in a fixed order (slabs
// of 64 rows, then the slabs in order), so a measurement's result does not
// depend on scheduling; with unit (or dyadic) weights every bin is an exact
// sum, bit-equal to the reference's running sums.  The block's close (the
// reference's stop_block) runs on the host once per block.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "alea_estimators.h"

namespace alea_gpu {

namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr size_t kPartBudget = size_t(32) << 20;   // bytes of per-row partial sums, all chains
constexpr int kSmemRowDoubles = 5120;               // rows up to 40 KB are staged in shared memory
constexpr int kRowsTarget = 148 * 32;               // warps in flight: 32 one-warp CTAs per SM

struct EstLaunch {
    const double* rec;       // walker records or compact position rows
    long stride;
    int o_pos, o_w;
    const int* idx;          // configuration c is block idx[c] (null: c)
    const double* weights;   // [nw], or null: the blocks' weights
    int unit;                // every weight 1
    int nw, chains, rows;
    double* part;            // [chains * rows][width1]
    int width1;              // sums of one row + the weight sum
    int smem_row;            // the row lives in shared memory
};

// Walkers [w0, w1) of row r of chain t: chains are the even contiguous split
// of the population that VMC's streams use, rows even splits of a chain.
__device__ __forceinline__ void row_range(const EstLaunch& L, int t, int r, int& w0, int& w1) {
    const int base = L.nw / L.chains, rem = L.nw % L.chains;
    const int c0 = t * base + min(t, rem), cn = base + (t < rem ? 1 : 0);
    const int rb = cn / L.rows, rr = cn % L.rows;
    w0 = c0 + r * rb + min(r, rr);
    w1 = w0 + rb + (r < rr ? 1 : 0);
}

__device__ __forceinline__ long block_of_conf(const EstLaunch& L, int w) { return L.idx ? L.idx[w] : w; }

__device__ __forceinline__ double weight_of(const EstLaunch& L, int w) {
    if (L.unit) return 1.0;
    if (L.weights) return L.weights[w];
    return L.rec[block_of_conf(L, w) * L.stride + L.o_w];
}

__device__ __forceinline__ double* row_of(const EstLaunch& L, double* smem_row) {
    return L.smem_row ? smem_row
                      : L.part + (static_cast<long>(blockIdx.y) * L.rows + blockIdx.x) * L.width1;
}

__device__ __forceinline__ void row_zero(const EstLaunch& L, double* row) {
    for (int k = threadIdx.x; k < L.width1; k += 32) row[k] = 0.0;
    __syncwarp();
}

__device__ __forceinline__ void row_flush(const EstLaunch& L, const double* row) {
    __syncwarp();
    if (!L.smem_row) return;
    double* dst = L.part + (static_cast<long>(blockIdx.y) * L.rows + blockIdx.x) * L.width1;
    for (int k = threadIdx.x; k < L.width1; k += 32) dst[k] = row[k];
}

// row[idx] += wt × (lanes holding idx), once per distinct idx >= 0.
__device__ __forceinline__ void add_binned(double* row, int idx, double wt) {
    const unsigned peers = __match_any_sync(kAll, idx);
    if (idx >= 0 && static_cast<int>(threadIdx.x) == __ffs(peers) - 1)
        row[idx] += wt * static_cast<double>(__popc(peers));
    __syncwarp();
}

// Triangular index of the unordered group pair (pair_correlation.cpp:88-93).
__device__ __forceinline__ int pair_id(int ga, int gb, int ng) {
    if (gb < ga) {
        const int t = ga;
        ga = gb;
        gb = t;
    }
    return ga * ng - ga * (ga - 1) / 2 + (gb - ga);
}

// Group of particle p from the group ranges (kernel parameters, no load).
__device__ __forceinline__ int group_at(const DevSys& s, int p) {
    int g = 0;
    for (int q = 0; q < s.ngroups; ++q)
        if (p >= s.gfirst[q] && p < s.glast[q]) g = q;
    return g;
}

// PairCorrelation::accumulate (pair_correlation.cpp:99-127): every pair i < j
// at its minimum-image distance |r_i - r_j| (the distance table's value,
// batched_distance_table.cpp:20-55), binned below rmax.  A walker's pairs are
// first counted per bin (integer shared-memory atomics: exact, order-free);
// then each bin with a count adds weight × count to the row once.  The pair
// list is staged in shared memory when pairs_smem is set.
__global__ void __launch_bounds__(32) gofr_kernel(const __grid_constant__ DevSys s, const EstLaunch L,
                                                  const int2* __restrict__ pairs, int npair, int pairs_smem,
                                                  double rmax, double inv_delta, int n_bins) {
    extern __shared__ double sm[];
    const int width = L.width1 - 1;
    double* pos = sm;                                           // [np * 2]
    int* cnt = reinterpret_cast<int*>(pos + ((s.np * 2 + 1) & ~1));   // [width]
    int2* spairs = reinterpret_cast<int2*>(cnt + ((width + 1) & ~1));
    double* row = row_of(L, reinterpret_cast<double*>(spairs + (pairs_smem ? npair : 0)));
    const int lane = threadIdx.x;
    const int2* pt = pairs;
    if (pairs_smem) {
        for (int q = lane; q < npair; q += 32) spairs[q] = pairs[q];
        pt = spairs;
    }
    for (int k = lane; k < width; k += 32) cnt[k] = 0;
    row_zero(L, row);
    int w0, w1;
    row_range(L, blockIdx.y, blockIdx.x, w0, w1);
    for (int w = w0; w < w1; ++w) {
        const double* r = L.rec + block_of_conf(L, w) * L.stride + L.o_pos;
        for (int k = lane; k < s.np * 2; k += 32) pos[k] = r[k];
        const double wt = weight_of(L, w);
        __syncwarp();
        for (int q = lane; q < npair; q += 32) {
            const int2 ij = pt[q];
            double dx, dy;
            const double d = fold2(s, pos[ij.x * 2], pos[ij.x * 2 + 1], pos[ij.y * 2], pos[ij.y * 2 + 1], dx, dy);
            if (d < rmax) {
                const unsigned long long bin = static_cast<unsigned long long>(d * inv_delta);
                if (bin < static_cast<unsigned long long>(n_bins))
                    atomicAdd(cnt + pair_id(group_at(s, ij.x), group_at(s, ij.y), s.ngroups) * n_bins +
                                  static_cast<int>(bin),
                              1);
            }
        }
        __syncwarp();
        for (int k = lane; k < width; k += 32) {
            const int c = cnt[k];
            if (c) {
                row[k] += wt * static_cast<double>(c);
                cnt[k] = 0;
            }
        }
        if (lane == 0) row[width] += wt;
        __syncwarp();
    }
    row_flush(L, row);
}

__device__ __forceinline__ int grid_bin(double x, int n_bins) {
    unsigned long long b = static_cast<unsigned long long>(x * static_cast<double>(n_bins));
    if (b >= static_cast<unsigned long long>(n_bins)) b = n_bins - 1;   // rounding at the upper edge
    return static_cast<int>(b);
}

// Density::accumulate (density.cpp:70-130): a periodic cell bins the
// fractional coordinates of the wrapped position on the n_bins² grid tiling
// the cell; an open one the box [-rmax, rmax)², dropping particles outside.
__global__ void __launch_bounds__(32) density_kernel(const __grid_constant__ DevSys s, const EstLaunch L,
                                                     double rmax, int n_bins, int per_particle) {
    extern __shared__ double sm[];
    double* row = row_of(L, sm);
    row_zero(L, row);
    int w0, w1;
    row_range(L, blockIdx.y, blockIdx.x, w0, w1);
    const int lane = threadIdx.x;
    const int n_cells = n_bins * n_bins;
    const double two_rmax = 2.0 * rmax, inv_delta = static_cast<double>(n_bins) / (2.0 * rmax);
    for (int w = w0; w < w1; ++w) {
        const double* r = L.rec + block_of_conf(L, w) * L.stride + L.o_pos;
        const double wt = weight_of(L, w);
        for (int p0 = 0; p0 < s.np; p0 += 32) {
            const int p = p0 + lane;
            int idx = -1;
            if (p < s.np) {
                double x = r[p * 2], y = r[p * 2 + 1];
                const int ser = per_particle ? p : s.group_of[p];
                if (s.periodic) {
                    wrap2(s, x, y);
                    const double f0 = fma(s.ainv[1], y, s.ainv[0] * x);
                    const double f1 = fma(s.ainv[3], y, s.ainv[2] * x);
                    idx = ser * n_cells + grid_bin(f0 + 0.5, n_bins) * n_bins + grid_bin(f1 + 0.5, n_bins);
                } else {
                    const double xs = x + rmax, ys = y + rmax;
                    if (xs >= 0.0 && xs < two_rmax && ys >= 0.0 && ys < two_rmax) {
                        int b0 = static_cast<int>(xs * inv_delta), b1 = static_cast<int>(ys * inv_delta);
                        b0 = min(b0, n_bins - 1);
                        b1 = min(b1, n_bins - 1);
                        idx = ser * n_cells + b0 * n_bins + b1;
                    }
                }
            }
            add_binned(row, idx, wt);
        }
        if (lane == 0) row[L.width1 - 1] += wt;
        __syncwarp();
    }
    row_flush(L, row);
}

// Cell of particle p of a walker for the density grid (as density_kernel), or
// -1 outside an open cell's box.
__device__ __forceinline__ int density_cell(const DevSys& s, double x, double y, double rmax, int n_bins) {
    if (s.periodic) {
        wrap2(s, x, y);
        const double f0 = fma(s.ainv[1], y, s.ainv[0] * x);
        const double f1 = fma(s.ainv[3], y, s.ainv[2] * x);
        return grid_bin(f0 + 0.5, n_bins) * n_bins + grid_bin(f1 + 0.5, n_bins);
    }
    const double two_rmax = 2.0 * rmax, inv_delta = static_cast<double>(n_bins) / (2.0 * rmax);
    const double xs = x + rmax, ys = y + rmax;
    if (!(xs >= 0.0 && xs < two_rmax && ys >= 0.0 && ys < two_rmax)) return -1;
    const int b0 = min(static_cast<int>(xs * inv_delta), n_bins - 1);
    const int b1 = min(static_cast<int>(ys * inv_delta), n_bins - 1);
    return b0 * n_bins + b1;
}

// The per-particle density (one series per particle): one warp per
// (walker range r, particle p, chain t) keeps only particle p's grid, its
// lanes taking 32 walkers at a time; lanes in one cell are grouped with
// match.any and their leader adds their weights summed in lane order.  The
// p = 0 warps also sum the weights.  Output: the warp's row in
// part[((t * np + p) * ranges + r)][n_cells + 1].
__global__ void __launch_bounds__(32) density_pp_kernel(const __grid_constant__ DevSys s, const EstLaunch L,
                                                        double rmax, int n_bins) {
    extern __shared__ double sm[];
    const int n_cells = n_bins * n_bins, width1 = n_cells + 1;
    const int r = blockIdx.x, p = blockIdx.y, t = blockIdx.z, lane = threadIdx.x;
    double* row = sm;
    for (int k = lane; k < width1; k += 32) row[k] = 0.0;
    __syncwarp();
    int w0, w1;
    row_range(L, t, r, w0, w1);
    for (int base = w0; base < w1; base += 32) {
        const int w = base + lane;
        int idx = -1;
        double wt = 0.0;
        if (w < w1) {
            wt = weight_of(L, w);
            const double* rp = L.rec + block_of_conf(L, w) * L.stride + L.o_pos;
            idx = density_cell(s, rp[p * 2], rp[p * 2 + 1], rmax, n_bins);
        }
        const unsigned peers = __match_any_sync(kAll, idx);
        double sum = 0.0, tw = 0.0;
        for (int q = 0; q < 32; ++q) {
            const double wq = __shfl_sync(kAll, wt, q);
            if ((peers >> q) & 1u) sum += wq;
            tw += wq;
        }
        if (idx >= 0 && lane == __ffs(peers) - 1) row[idx] += sum;
        if (p == 0 && lane == 0) row[n_cells] += tw;
        __syncwarp();
    }
    double* dst = L.part + ((static_cast<long>(t) * gridDim.y + p) * gridDim.x + r) * width1;
    for (int k = lane; k < width1; k += 32) dst[k] = row[k];
}

// e^{inθ}, n = 0..m, by ReciprocalPhases' recurrence
// (src/numerics/reciprocal_phases.h:62-76), into lad[2n], lad[2n + 1].
__device__ __forceinline__ void ladder(double theta, int m, double* lad) {
    double c, sn;
    sincos(theta, &sn, &c);
    double re = 1.0, im = 0.0;
    lad[0] = 1.0;
    lad[1] = 0.0;
    for (int n = 1; n <= m; ++n) {
        const double r2 = fma(re, c, -(im * sn));
        const double i2 = fma(re, sn, im * c);
        re = r2;
        im = i2;
        lad[2 * n] = re;
        lad[2 * n + 1] = im;
    }
}

__device__ __forceinline__ void pick(const double* lad, int n, double& re, double& im) {
    const int a = n < 0 ? -n : n;
    re = lad[2 * a];
    im = n < 0 ? -lad[2 * a + 1] : lad[2 * a + 1];
}

// ρ(k) += Σ_q e^{ik·r_q} over the cnt particles whose ladders are in lad, for
// this lane's NS k-vectors k = 32 (c0 + c) + lane; the NS sums are independent
// chains, particles in order within each.
template <int NS>
__device__ __forceinline__ void rho_slots(const int* __restrict__ kn, int nk, int c0, const double* lad, int lw,
                                          int m1, int cnt, double* re, double* im) {
    const int lane = threadIdx.x;
    int a[NS], b[NS];
    double sr[NS], si[NS];
#pragma unroll
    for (int c = 0; c < NS; ++c) {
        const int k = (c0 + c) * 32 + lane;
        const bool in = k < nk;
        a[c] = in ? kn[k] : 0;
        b[c] = in ? kn[nk + k] : 0;
        sr[c] = in ? re[k] : 0.0;
        si[c] = in ? im[k] : 0.0;
    }
    for (int q = 0; q < cnt; ++q) {
        const double* l1 = lad + q * lw;
        const double* l2 = l1 + 2 * (m1 + 1);
#pragma unroll
        for (int c = 0; c < NS; ++c) {
            double ar, ai, br, bi;
            pick(l1, a[c], ar, ai);
            pick(l2, b[c], br, bi);
            sr[c] += ar * br - ai * bi;
            si[c] += ar * bi + ai * br;
        }
    }
#pragma unroll
    for (int c = 0; c < NS; ++c) {
        const int k = (c0 + c) * 32 + lane;
        if (k < nk) {
            re[k] = sr[c];
            im[k] = si[c];
        }
    }
}

// StructureFactor::accumulate (structure_factor.cpp:80-121): per walker the
// group densities ρ_g(k) = Σ_{i∈g} e^{ik·r_i}, then per k (one lane each)
// Re ρ_g, Im ρ_g and, for every group pair a <= b, Re ρ_a Re ρ_b + Im ρ_a
// Im ρ_b, times the weight.  A group's particles are taken 32 at a time: each
// lane builds its particle's two ladders, then each lane sums its k-vectors
// over the 32 particles in particle order.
// Row: [pair][k] S sums, [group][k] Re ρ, [group][k] Im ρ, W.
__global__ void __launch_bounds__(32) sofk_kernel(const __grid_constant__ DevSys s, const EstLaunch L,
                                                  const int* __restrict__ kn, int nk, int m1, int m2) {
    extern __shared__ double sm[];
    const int ng = s.ngroups, lane = threadIdx.x;
    const int npairs = ng * (ng + 1) / 2;
    const int lw = 2 * (m1 + 1) + 2 * (m2 + 1);         // one particle's two ladders
    double* rho = sm;                                   // [ng][2][nk]
    double* lad = rho + 2 * ng * nk;                    // [32][lw]
    double* row = row_of(L, lad + 32 * lw);
    row_zero(L, row);
    int w0, w1;
    row_range(L, blockIdx.y, blockIdx.x, w0, w1);
    for (int w = w0; w < w1; ++w) {
        const double* r = L.rec + block_of_conf(L, w) * L.stride + L.o_pos;
        const double wt = weight_of(L, w);
        for (int k = lane; k < 2 * ng * nk; k += 32) rho[k] = 0.0;
        for (int g = 0; g < ng; ++g) {
            double* re = rho + 2 * g * nk;
            double* im = re + nk;
            for (int i0 = s.gfirst[g]; i0 < s.glast[g]; i0 += 32) {
                const int cnt = min(32, s.glast[g] - i0);
                __syncwarp();   // rho zeroed, the previous particles' ladders read
                if (lane < cnt) {
                    const double x = r[(i0 + lane) * 2], y = r[(i0 + lane) * 2 + 1];
                    ladder(s.recip[0] * x + s.recip[1] * y, m1, lad + lane * lw);
                    ladder(s.recip[2] * x + s.recip[3] * y, m2, lad + lane * lw + 2 * (m1 + 1));
                }
                __syncwarp();
                const int slots = (nk + 31) / 32;
                for (int c0 = 0; c0 < slots; c0 += 4) {
                    switch (min(slots - c0, 4)) {
                        case 1: rho_slots<1>(kn, nk, c0, lad, lw, m1, cnt, re, im); break;
                        case 2: rho_slots<2>(kn, nk, c0, lad, lw, m1, cnt, re, im); break;
                        case 3: rho_slots<3>(kn, nk, c0, lad, lw, m1, cnt, re, im); break;
                        default: rho_slots<4>(kn, nk, c0, lad, lw, m1, cnt, re, im); break;
                    }
                }
            }
        }
        for (int k = lane; k < nk; k += 32) {
            for (int g = 0; g < ng; ++g) {
                row[(npairs + g) * nk + k] += wt * rho[2 * g * nk + k];
                row[(npairs + ng + g) * nk + k] += wt * rho[(2 * g + 1) * nk + k];
            }
            int pid = 0;
            for (int a = 0; a < ng; ++a)
                for (int b = a; b < ng; ++b, ++pid) {
                    const double ra = rho[2 * a * nk + k], ia = rho[(2 * a + 1) * nk + k];
                    const double rb = rho[2 * b * nk + k], ib = rho[(2 * b + 1) * nk + k];
                    row[pid * nk + k] += wt * fma(ra, rb, ia * ib);
                }
        }
        if (lane == 0) row[L.width1 - 1] += wt;
        __syncwarp();
    }
    row_flush(L, row);
}

constexpr int kSlab = 64;   // rows summed by one CTA of the first reduction stage

// First stage: slab j of chain t (rows [64 j, 64 j + 64)) summed per column.
// Thread (warp v, lane l) takes column k = 32 x + l and adds rows
// 64 j + v + 8 i in i order; the 8 warps' sums are added in warp order.
__global__ void __launch_bounds__(256) est_slab_kernel(const double* __restrict__ part, int rows, int width1,
                                                       int slabs, double* __restrict__ part2) {
    __shared__ double red[8][32];
    const int l = threadIdx.x & 31, v = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + l, j = blockIdx.y, t = blockIdx.z;
    double sum = 0.0;
    if (k < width1) {
        const double* p = part + static_cast<long>(t) * rows * width1 + k;
        const int r1 = min(rows, (j + 1) * kSlab);
#pragma unroll 4
        for (int q = j * kSlab + v; q < r1; q += 8) sum += p[static_cast<long>(q) * width1];
    }
    red[v][l] = sum;
    __syncthreads();
    if (v == 0 && k < width1) {
        double a = red[0][l];
        for (int q = 1; q < 8; ++q) a += red[q][l];
        part2[(static_cast<long>(t) * slabs + j) * width1 + k] = a;
    }
}

// The per-particle density's rows into the running block: acc[t][p n_cells + c]
// += Σ_r part[t][p][r][c] in range order, and W from the p = 0 rows.
__global__ void est_pp_sum_kernel(const double* __restrict__ part, int ranges, int np, int n_cells, int chains,
                                  double* __restrict__ acc) {
    const long width1 = n_cells + 1;
    const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (e >= static_cast<long>(chains) * np * width1) return;
    const long t = e / (np * width1), rem = e % (np * width1);
    const long p = rem / width1, c = rem % width1;
    if (c == n_cells && p != 0) return;
    const double* src = part + (t * np + p) * ranges * width1 + c;
    double a = 0.0;
    for (int q = 0; q < ranges; ++q) a += src[static_cast<long>(q) * width1];
    double* dst = acc + t * (static_cast<long>(np) * n_cells + 1);
    if (c < n_cells) dst[p * n_cells + c] += a;
    else dst[static_cast<long>(np) * n_cells] += a;
}

// Second stage: acc[t][k] += Σ_j part2[t][j][k], slabs in order.
__global__ void est_sum_kernel(const double* __restrict__ part2, int slabs, int width1, int chains,
                               double* __restrict__ acc) {
    const long e = blockIdx.x * static_cast<long>(blockDim.x) + threadIdx.x;
    if (e >= static_cast<long>(chains) * width1) return;
    const long t = e / width1, k = e % width1;
    const double* p = part2 + t * slabs * width1 + k;
    double a = 0.0;
    for (int j = 0; j < slabs; ++j) a += p[static_cast<long>(j) * width1];
    acc[e] += a;
}

}  // namespace

// ───────────────────────── host side ───────────────────────────────────

struct DevEstimator {
    alea_gpu_estimator_spec spec{};
    int width = 0;                 // running sums per chain (without W)
    int out_width = 0;             // doubles per block estimate
    int n_series = 0, n_cells = 0, nk = 0, ns = 0;
    double inv_delta = 0.0, volume = 0.0, cell_volume = 0.0;
    std::vector<double> group_n;   // particles per group
    std::vector<int> n1, n2, shell_of, shell_count;
    std::vector<double> kx, ky, shell_k;
    int m1 = 0, m2 = 0;
    int* d_kn = nullptr;           // n1 | n2
    double* d_acc = nullptr;       // [chains][width + 1]
    std::vector<std::vector<double>> hist;   // per chain: blocks × out_width
    int n_blocks = 0;
};

struct EstimatorSet {
    std::vector<DevEstimator> e;
    double* d_part = nullptr;      // per-row sums of one measurement
    size_t part_bytes = 0;
    double* d_part2 = nullptr;     // per-slab sums
    size_t part2_bytes = 0;
    int chains = 0;
};

namespace {

void free_one(DevEstimator& d, cudaStream_t st) {
    if (d.d_kn) cudaFreeAsync(d.d_kn, st);
    if (d.d_acc) cudaFreeAsync(d.d_acc, st);
    d.d_kn = nullptr;
    d.d_acc = nullptr;
}

double ws_radius(const DevSys& s) {
    // half the shortest nonzero lattice vector over a ±2 window
    // (simulation_cell.cpp:202-224)
    double best = 0.0;
    for (int n0 = -2; n0 <= 2; ++n0)
        for (int n1 = -2; n1 <= 2; ++n1) {
            if (n0 == 0 && n1 == 0) continue;
            const double x = n0 * s.a[0] + n1 * s.a[2], y = n0 * s.a[1] + n1 * s.a[3];
            const double r2 = x * x + y * y;
            if (best == 0.0 || r2 < best) best = r2;
        }
    return 0.5 * std::sqrt(best);
}

}  // namespace

int est_add(EstimatorSet*& set, const DevSys& s, const alea_gpu_estimator_spec& spec, cudaStream_t st,
            std::string& err, int* id) {
    if (s.dim != 2) {
        err = "estimators: the walker records hold 2-D positions";
        return ALEA_ERR_UNSUPPORTED;
    }
    DevEstimator d;
    d.spec = spec;
    const int ng = s.ngroups;
    d.volume = s.periodic ? std::abs(s.a[0] * s.a[3] - s.a[1] * s.a[2]) : 0.0;
    for (int g = 0; g < ng; ++g) d.group_n.push_back(s.glast[g] - s.gfirst[g]);
    if (spec.kind == ALEA_EST_GOFR) {
        if (spec.n_bins < 1 || !(spec.rmax > 0.0)) {
            err = "gofr: n_bins >= 1 and rmax > 0 are needed";
            return ALEA_ERR_INVALID;
        }
        if (s.periodic && spec.rmax > ws_radius(s)) {
            err = "gofr rmax " + std::to_string(spec.rmax) + " exceeds the cell's Wigner-Seitz inradius " +
                  std::to_string(ws_radius(s)) + "; minimum-image distances are not unique beyond it";
            return ALEA_ERR_INVALID;
        }
        d.n_series = ng * (ng + 1) / 2;
        d.width = d.out_width = d.n_series * spec.n_bins;
        d.inv_delta = static_cast<double>(spec.n_bins) / spec.rmax;
    } else if (spec.kind == ALEA_EST_DENSITY) {
        if (spec.n_bins < 1 || spec.n_bins > 4096 || (!s.periodic && !(spec.rmax > 0.0))) {
            err = "density: 1 <= n_bins <= 4096 and, for an open cell, rmax > 0 are needed";
            return ALEA_ERR_INVALID;
        }
        d.n_cells = spec.n_bins * spec.n_bins;
        d.n_series = spec.per_particle ? s.np : ng;
        d.width = d.out_width = d.n_series * d.n_cells;
        const double delta = 2.0 * spec.rmax / spec.n_bins;
        d.cell_volume = s.periodic ? d.volume / d.n_cells : delta * delta;
    } else if (spec.kind == ALEA_EST_SOFK) {
        if (!s.periodic) {
            err = "sofk: the structure factor needs a periodic 2-D cell";
            return ALEA_ERR_INVALID;
        }
        // half-space k set (structure_factor.cpp:18-59)
        const double* b = s.recip;
        const double b1 = std::hypot(b[0], b[1]), b2 = std::hypot(b[2], b[3]);
        const int nmax = static_cast<int>(std::ceil(spec.kmax / std::min(b1, b2))) + 1;
        struct K {
            double k;
            int n1, n2;
            double kx, ky;
        };
        std::vector<K> ks;
        for (int i = 0; i <= nmax; ++i)
            for (int j = -nmax; j <= nmax; ++j) {
                if (i == 0 && j <= 0) continue;
                const double kx = i * b[0] + j * b[2], ky = i * b[1] + j * b[3];
                const double k = std::hypot(kx, ky);
                if (k <= spec.kmax) ks.push_back({k, i, j, kx, ky});
            }
        if (ks.empty()) {
            err = "sofk: kmax " + std::to_string(spec.kmax) + " is below the shortest reciprocal vector " +
                  std::to_string(std::min(b1, b2)) + " of the cell";
            return ALEA_ERR_INVALID;
        }
        std::stable_sort(ks.begin(), ks.end(), [](const K& x, const K& y) { return x.k < y.k; });
        const double tol = 1e-9 * std::min(b1, b2);
        for (const K& q : ks) {
            if (d.shell_k.empty() || q.k - d.shell_k.back() > tol) {
                d.shell_k.push_back(q.k);
                d.shell_count.push_back(0);
            }
            ++d.shell_count.back();
            d.shell_of.push_back(static_cast<int>(d.shell_k.size()) - 1);
            d.n1.push_back(q.n1);
            d.n2.push_back(q.n2);
            d.kx.push_back(q.kx);
            d.ky.push_back(q.ky);
            d.m1 = std::max(d.m1, std::abs(q.n1));
            d.m2 = std::max(d.m2, std::abs(q.n2));
        }
        d.nk = static_cast<int>(ks.size());
        d.ns = static_cast<int>(d.shell_k.size());
        d.n_series = ng * (ng + 1) / 2;
        d.width = (d.n_series + 2 * ng) * d.nk;
        d.out_width = d.n_series * d.ns + 2 * ng * d.nk;
        std::vector<int> kn(d.n1);
        kn.insert(kn.end(), d.n2.begin(), d.n2.end());
        if (cudaMallocAsync(&d.d_kn, kn.size() * sizeof(int), st) != cudaSuccess ||
            cudaMemcpyAsync(d.d_kn, kn.data(), kn.size() * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            free_one(d, st);
            err = "sofk: device allocation failed";
            return ALEA_ERR_NOMEM;
        }
    } else {
        err = "unknown estimator kind " + std::to_string(spec.kind);
        return ALEA_ERR_INVALID;
    }
    if (!set) set = new EstimatorSet();
    if (set->chains > 0) {   // measurements already run: join them with an empty block
        const size_t b = sizeof(double) * (d.width + 1) * set->chains;
        if (cudaMallocAsync(&d.d_acc, b, st) != cudaSuccess || cudaMemsetAsync(d.d_acc, 0, b, st) != cudaSuccess) {
            free_one(d, st);
            err = "estimators: device allocation failed";
            return ALEA_ERR_NOMEM;
        }
        d.hist.assign(set->chains, {});
    }
    set->e.push_back(std::move(d));
    *id = static_cast<int>(set->e.size()) - 1;
    return ALEA_OK;
}

void est_free(EstimatorSet*& set, cudaStream_t st) {
    if (!set) return;
    for (DevEstimator& d : set->e) free_one(d, st);
    if (set->d_part) cudaFreeAsync(set->d_part, st);
    if (set->d_part2) cudaFreeAsync(set->d_part2, st);
    delete set;
    set = nullptr;
}

int est_count(const EstimatorSet* set) { return set ? static_cast<int>(set->e.size()) : 0; }

int est_reset(EstimatorSet* set, cudaStream_t st, std::string& err) {
    if (!set) return ALEA_OK;
    for (DevEstimator& d : set->e) {
        if (d.d_acc) cudaFreeAsync(d.d_acc, st);
        d.d_acc = nullptr;
        d.hist.clear();
        d.n_blocks = 0;
    }
    set->chains = 0;
    (void)err;
    return ALEA_OK;
}

int est_start_block(EstimatorSet* set, cudaStream_t st, std::string& err) {
    if (!set || set->chains == 0) return ALEA_OK;   // zeroed when the chains are first set
    for (DevEstimator& d : set->e)
        if (cudaMemsetAsync(d.d_acc, 0, sizeof(double) * (d.width + 1) * set->chains, st) != cudaSuccess) {
            err = "estimators: cudaMemsetAsync failed";
            return ALEA_ERR_CUDA;
        }
    return ALEA_OK;
}

int est_accumulate(EstimatorSet* set, const DevSys& s, const EstSource& src, const double* d_weights, bool unit,
                   int chains, const int2* pairs, int npair, cudaStream_t st, std::string& err, uint64_t* launches) {
    if (!set || set->e.empty()) return ALEA_OK;
    const int nw = src.n;
    if (!unit && !d_weights && src.o_w < 0) {
        err = "estimators: the configurations carry no weights";
        return ALEA_ERR_INVALID;
    }
    if (chains < 1 || chains > nw || chains > 65535) {
        err = "estimators: n_chains must be in [1, min(walkers, 65535)]";
        return ALEA_ERR_INVALID;
    }
    if (set->chains == 0) {
        set->chains = chains;
        for (DevEstimator& d : set->e) {
            const size_t b = sizeof(double) * (d.width + 1) * chains;
            if (cudaMallocAsync(&d.d_acc, b, st) != cudaSuccess || cudaMemsetAsync(d.d_acc, 0, b, st) != cudaSuccess) {
                err = "estimators: device allocation failed";
                return ALEA_ERR_NOMEM;
            }
            d.hist.assign(chains, {});
        }
    } else if (chains != set->chains) {
        err = "estimators: the chain count changed without a reset (" + std::to_string(set->chains) + " -> " +
              std::to_string(chains) + ")";
        return ALEA_ERR_INVALID;
    }
    const int min_chain = nw / chains;
    auto ensure = [&](double** buf, size_t* have, size_t want) {
        if (want <= *have) return true;
        if (*buf) cudaFreeAsync(*buf, st);
        *buf = nullptr;
        *have = 0;
        if (cudaMallocAsync(buf, want, st) != cudaSuccess) return false;
        *have = want;
        return true;
    };
    // one binning launch's view of the source: `rows` walker ranges per chain,
    // each writing a row of `width1` sums into the scratch
    auto launch_of = [&](int rows, int width1) {
        EstLaunch L{};
        L.rec = src.base;
        L.stride = src.stride;
        L.o_pos = src.o_pos;
        L.o_w = src.o_w;
        L.idx = src.idx;
        L.weights = d_weights;
        L.unit = unit ? 1 : 0;
        L.nw = nw;
        L.chains = chains;
        L.rows = rows;
        L.part = set->d_part;
        L.width1 = width1;
        return L;
    };
    for (DevEstimator& d : set->e) {
        const int width1 = d.width + 1;
        const int cells1 = d.n_cells + 1;
        if (d.spec.kind == ALEA_EST_DENSITY && d.spec.per_particle && cells1 <= kSmemRowDoubles) {
            // one particle's grid per warp (density_pp_kernel); a group density
            // stays on density_kernel, whose one row per walker range is faster
            // there (0.067 against 0.137 ms at N = 42, 16,384 walkers)
            const size_t per = sizeof(double) * cells1 * s.np * chains;
            const int ranges = static_cast<int>(std::max<size_t>(
                1, std::min<size_t>({static_cast<size_t>((min_chain + 31) / 32), kPartBudget / per, 64})));
            if (!ensure(&set->d_part, &set->part_bytes, per * ranges)) {
                err = "estimators: device allocation failed";
                return ALEA_ERR_NOMEM;
            }
            const EstLaunch L = launch_of(ranges, cells1);
            density_pp_kernel<<<dim3(ranges, s.np, chains), 32, sizeof(double) * cells1, st>>>(s, L, d.spec.rmax,
                                                                                              d.spec.n_bins);
            const long n = static_cast<long>(chains) * s.np * cells1;
            est_pp_sum_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, st>>>(set->d_part, ranges, s.np,
                                                                                d.n_cells, chains, d.d_acc);
            if (launches) *launches += 2;
            if (cudaGetLastError() != cudaSuccess) {
                err = "estimators: kernel launch failed";
                return ALEA_ERR_CUDA;
            }
            continue;
        }
        int rows = std::max(1, std::min(min_chain, (kRowsTarget + chains - 1) / chains));
        const size_t per_row = sizeof(double) * width1;
        rows = static_cast<int>(std::max<size_t>(1, std::min<size_t>(rows, kPartBudget / (per_row * chains))));
        const size_t need = per_row * rows * chains;
        const int slabs = (rows + kSlab - 1) / kSlab;
        const size_t need2 = per_row * slabs * chains;
        if (!ensure(&set->d_part, &set->part_bytes, need) || !ensure(&set->d_part2, &set->part2_bytes, need2)) {
            err = "estimators: device allocation failed";
            return ALEA_ERR_NOMEM;
        }
        EstLaunch L = launch_of(rows, width1);
        L.smem_row = width1 <= kSmemRowDoubles ? 1 : 0;
        const dim3 grid(rows, chains);
        size_t smem = L.smem_row ? sizeof(double) * width1 : 0;
        const alea_gpu_estimator_spec& sp = d.spec;
        if (sp.kind == ALEA_EST_GOFR) {
            smem += sizeof(double) * ((s.np * 2 + 1) & ~1) + sizeof(int) * ((d.width + 1) & ~1);
            if (smem > 48 * 1024) {
                err = "gofr: too many bins for one warp's shared memory (" + std::to_string(d.width) + ")";
                return ALEA_ERR_UNSUPPORTED;
            }
            const int pairs_smem = smem + sizeof(int2) * npair <= 40 * 1024 ? 1 : 0;
            if (pairs_smem) smem += sizeof(int2) * npair;
            gofr_kernel<<<grid, 32, smem, st>>>(s, L, pairs, npair, pairs_smem, sp.rmax, d.inv_delta, sp.n_bins);
        } else if (sp.kind == ALEA_EST_DENSITY) {
            density_kernel<<<grid, 32, smem, st>>>(s, L, sp.rmax, sp.n_bins, sp.per_particle ? 1 : 0);
        } else {
            smem += sizeof(double) * (2 * s.ngroups * d.nk + 32 * (2 * (d.m1 + 1) + 2 * (d.m2 + 1)));
            if (smem > 48 * 1024) {
                err = "sofk: too many k-vectors for one warp's shared memory (n_k = " + std::to_string(d.nk) + ")";
                return ALEA_ERR_UNSUPPORTED;
            }
            sofk_kernel<<<grid, 32, smem, st>>>(s, L, d.d_kn, d.nk, d.m1, d.m2);
        }
        est_slab_kernel<<<dim3((width1 + 31) / 32, slabs, chains), 256, 0, st>>>(set->d_part, rows, width1, slabs,
                                                                                set->d_part2);
        const long n = static_cast<long>(chains) * width1;
        est_sum_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, st>>>(set->d_part2, slabs, width1, chains,
                                                                         d.d_acc);
        if (launches) *launches += 3;
        if (cudaGetLastError() != cudaSuccess) {
            err = "estimators: kernel launch failed";
            return ALEA_ERR_CUDA;
        }
    }
    return ALEA_OK;
}

int est_stop_block(EstimatorSet* set, cudaStream_t st, std::string& err, uint64_t* d2h) {
    if (!set || set->e.empty()) return ALEA_OK;
    if (set->chains == 0) {
        err = "estimators: a block closed before any measurement";
        return ALEA_ERR_INVALID;
    }
    const int T = set->chains;
    for (DevEstimator& d : set->e) {
        const int width1 = d.width + 1;
        std::vector<double> acc(static_cast<size_t>(width1) * T);
        if (cudaMemcpyAsync(acc.data(), d.d_acc, sizeof(double) * acc.size(), cudaMemcpyDeviceToHost, st) !=
                cudaSuccess ||
            cudaMemsetAsync(d.d_acc, 0, sizeof(double) * acc.size(), st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            err = "estimators: reading the block back failed";
            return ALEA_ERR_CUDA;
        }
        if (d2h) *d2h += sizeof(double) * acc.size();
        for (int t = 0; t < T; ++t) {
            const double* h = acc.data() + static_cast<size_t>(t) * width1;
            const double W = h[d.width];
            std::vector<double> blk(d.out_width, 0.0);
            if (d.spec.kind == ALEA_EST_GOFR) {
                // pair_correlation.cpp:143-160
                if (W > 0.0) {
                    const double inv_w = 1.0 / W;
                    for (int k = 0; k < d.width; ++k) blk[k] = h[k] * inv_w;
                }
            } else if (d.spec.kind == ALEA_EST_DENSITY) {
                // density.cpp:153-170
                const double norm = W > 0.0 ? 1.0 / (W * d.cell_volume) : 0.0;
                for (int k = 0; k < d.width; ++k) blk[k] = h[k] * norm;
            } else if (W > 0.0) {
                // structure_factor.cpp:133-150
                const double inv_w = 1.0 / W;
                const int ng = static_cast<int>(d.group_n.size()), nk = d.nk, ns = d.ns;
                int pid = 0;
                for (int a = 0; a < ng; ++a)
                    for (int b = a; b < ng; ++b, ++pid) {
                        const double na = d.group_n[a], nb = d.group_n[b];
                        const double norm = (na > 0 && nb > 0) ? 1.0 / std::sqrt(na * nb) : 0.0;
                        for (int k = 0; k < nk; ++k)
                            blk[pid * ns + d.shell_of[k]] +=
                                h[pid * nk + k] * inv_w * norm / static_cast<double>(d.shell_count[d.shell_of[k]]);
                    }
                const int npairs = d.n_series;
                for (int q = 0; q < 2 * ng * nk; ++q) blk[npairs * ns + q] = h[npairs * nk + q] * inv_w;
            }
            d.hist[t].insert(d.hist[t].end(), blk.begin(), blk.end());
        }
        ++d.n_blocks;
    }
    return ALEA_OK;
}

int est_info(const EstimatorSet* set, int id, alea_gpu_estimator_desc* out) {
    if (!set || id < 0 || id >= static_cast<int>(set->e.size()) || !out) return ALEA_ERR_INVALID;
    const DevEstimator& d = set->e[id];
    *out = alea_gpu_estimator_desc{};
    out->kind = d.spec.kind;
    out->block_width = d.out_width;
    out->n_chains = set->chains;
    out->n_blocks = d.n_blocks;
    out->n_series = d.n_series;
    out->n_bins = d.spec.n_bins;
    out->n_cells = d.n_cells;
    out->n_k = d.nk;
    out->n_shells = d.ns;
    out->volume = d.volume;
    out->cell_volume = d.cell_volume;
    return ALEA_OK;
}

int est_blocks(const EstimatorSet* set, int id, double* out) {
    if (!set || id < 0 || id >= static_cast<int>(set->e.size()) || !out) return ALEA_ERR_INVALID;
    const DevEstimator& d = set->e[id];
    size_t o = 0;
    for (const auto& h : d.hist) {
        std::memcpy(out + o, h.data(), sizeof(double) * h.size());
        o += h.size();
    }
    return ALEA_OK;
}

int est_kvectors(const EstimatorSet* set, int id, int* n1, int* n2, double* kx, double* ky, int* shell_of,
                 double* shell_k, int* shell_count) {
    if (!set || id < 0 || id >= static_cast<int>(set->e.size())) return ALEA_ERR_INVALID;
    const DevEstimator& d = set->e[id];
    if (d.spec.kind != ALEA_EST_SOFK) return ALEA_ERR_INVALID;
    if (n1) std::copy(d.n1.begin(), d.n1.end(), n1);
    if (n2) std::copy(d.n2.begin(), d.n2.end(), n2);
    if (kx) std::copy(d.kx.begin(), d.kx.end(), kx);
    if (ky) std::copy(d.ky.begin(), d.ky.end(), ky);
    if (shell_of) std::copy(d.shell_of.begin(), d.shell_of.end(), shell_of);
    if (shell_k) std::copy(d.shell_k.begin(), d.shell_k.end(), shell_k);
    if (shell_count) std::copy(d.shell_count.begin(), d.shell_count.end(), shell_count);
    return ALEA_OK;
}

}  // namespace alea_gpu
