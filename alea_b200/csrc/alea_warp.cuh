// Device helpers of the one-warp sweeps (alea_fast.cu in FP64, alea_fast32.cu
// in the FP32 form): lane-slot utilities, 2-D orbitals, the warp
// Gauss-Jordan, the compact shared-memory layout and its record copies, and
// the local energy after a sweep.
#pragma once

#include "alea_walker.cuh"

namespace alea_gpu {

namespace {

// k-space contribution of one k to the gradient/Laplacian of a particle with
// phase (c, sn) that sees the density (pr, pi) (kspace_pair_sum.cpp:76-97).
__device__ __forceinline__ void kterm_r(double kx, double ky, double w, double c, double sn, double pr,
                                        double pi, double self, double* acc) {
    const double g = 2.0 * w * (c * pi - sn * pr);
    const double l = 2.0 * w * (self - (c * pr + sn * pi));
    acc[0] += kx * g;
    acc[1] += ky * g;
    acc[2] += kx * kx * l;
    acc[3] += ky * ky * l;
}

// Orbital rows ∇D, ∇²D of particle p (its block's row), lane slot j = column
// l + 32j; nothing for a particle outside every determinant.
template <int S>
__device__ __forceinline__ void fetch_rows(const DevSys& s, const double* grec, int p, double2 (&dg)[S],
                                           double2 (&dl)[S]) {
    const int b = block_of(s, p);
    if (b < 0) return;
    const DevBlock& B = s.blocks[b];
    const int N = B.n, kr = p - B.first;
    const double2* rg = reinterpret_cast<const double2*>(grec + B.oDg) + kr * N;
    const double2* rl = reinterpret_cast<const double2*>(grec + B.oDl) + kr * N;
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int m = static_cast<int>(threadIdx.x) + 32 * j;
        if (m < N) {
            dg[j] = __ldcg(rg + m);
            dl[j] = __ldcg(rl + m);
        }
    }
}

// Orbital i of a real block at (x, y): value, gradient, diagonal second
// derivatives (plane waves, orbital_set.h:436-474; Gaussians, :185-224).
__device__ __forceinline__ void orbital2(const DevSys& s, const DevBlock& B, int i, double x, double y,
                                         double& val, double& gx, double& gy, double& lx, double& ly) {
    if (B.type == 0) {
        const double k0 = B.k[i * 2], k1 = B.k[i * 2 + 1];
        double sn, c;
        sincos(fma(k1, y, k0 * x), &sn, &c);
        if (B.is_sin[i] != 0.0) {
            val = sn;
            gx = k0 * c;
            gy = k1 * c;
            lx = -k0 * k0 * sn;
            ly = -k1 * k1 * sn;
        } else {
            val = c;
            gx = -k0 * sn;
            gy = -k1 * sn;
            lx = -k0 * k0 * c;
            ly = -k1 * k1 * c;
        }
    } else {
        const double alpha = B.alphas[i];
        double dx = x - B.centers[i * 2], dy = y - B.centers[i * 2 + 1];
        min_image2(s, dx, dy);
        const double phi = exp(-alpha * fma(dy, dy, dx * dx));
        val = phi;
        gx = phi * (-2.0 * alpha * dx);
        gy = phi * (-2.0 * alpha * dy);
        lx = phi * (4.0 * alpha * alpha * dx * dx - 2.0 * alpha);
        ly = phi * (4.0 * alpha * alpha * dy * dy - 2.0 * alpha);
    }
}

// D (8x8) += A (8x4, row-major) B (4x8, column-major) on the FP64 tensor
// cores (mma.sync m8n8k4 .f64).  Lane l = 4g + t holds a = A[g][t],
// b = B[t][g] and d = D[g][2t], D[g][2t + 1].
__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// One Newton-Schulz step X <- X (2I - D X) of an inverse X (shared memory,
// row-major, stride N) against the block's orbital rows D (the record, row
// major), N <= 24, on the FP64 tensor cores: T = D X as 3 x 3 tiles of 8 x 8
// in registers, Y = 2I - T, then X Y tile row by tile row, each written back
// over the rows of X it was made from.  The residual of X after a run of
// Sherman-Morrison updates is ~1e-13, so one step leaves X = D⁻¹ to
// rounding, the inverse the Gauss-Jordan recomputation would give.  Returns
// max |T - I| (X untouched when it is not below 1e-6: the caller then
// recomputes by Gauss-Jordan).
__device__ double ns_refresh_warp(double* X, const double* D, int N) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int nb = (N + 7) >> 3;
    double y[3][3][2];
#pragma unroll
    for (int mt = 0; mt < 3; ++mt) {
        // this tile row's D fragments, all loads in flight before the products
        double a[6];
#pragma unroll
        for (int kt = 0; kt < 6; ++kt) {
            const int ar = mt * 8 + g, ac = kt * 4 + t;
            a[kt] = (mt < nb && ar < N && ac < N) ? D[ar * N + ac] : 0.0;
        }
#pragma unroll
        for (int nt = 0; nt < 3; ++nt) {
            y[mt][nt][0] = y[mt][nt][1] = 0.0;
            if (mt >= nb || nt >= nb) continue;
#pragma unroll
            for (int kt = 0; kt < 6; ++kt) {
                if (kt * 4 >= N) break;
                const int br = kt * 4 + t, bc = nt * 8 + g;
                const double b = (br < N && bc < N) ? X[br * N + bc] : 0.0;
                dmma_m8n8k4(y[mt][nt], a[kt], b);
            }
        }
    }
    double res = 0.0;
#pragma unroll
    for (int mt = 0; mt < 3; ++mt)
#pragma unroll
        for (int nt = 0; nt < 3; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = mt * 8 + g, col = nt * 8 + 2 * t + i;
                const bool in = row < N && col < N;
                const double id = row == col ? 1.0 : 0.0;
                if (in) res = fmax(res, fabs(y[mt][nt][i] - id));
                y[mt][nt][i] = in ? 2.0 * id - y[mt][nt][i] : 0.0;
            }
    res = warp_max(res);
    if (!(res < 1e-6)) return res;
#pragma unroll
    for (int mt = 0; mt < 3; ++mt) {
        if (mt >= nb) break;
        double o[3][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
        for (int nt = 0; nt < 3; ++nt) {
            if (nt >= nb) continue;
#pragma unroll
            for (int kt = 0; kt < 6; ++kt) {
                if (kt * 4 >= N) break;
                const int ar = mt * 8 + g, ac = kt * 4 + t;
                const double a = (ar < N && ac < N) ? X[ar * N + ac] : 0.0;
                // Y[kt*4 + t][nt*8 + g] from the lane holding it in its C fragment
                const int src = ((kt & 1) * 4 + t) * 4 + (g >> 1);
                const double b0 = __shfl_sync(kAllLanes, y[kt >> 1][nt][0], src);
                const double b1 = __shfl_sync(kAllLanes, y[kt >> 1][nt][1], src);
                dmma_m8n8k4(o[nt], a, (g & 1) ? b1 : b0);
            }
        }
        __syncwarp();
#pragma unroll
        for (int nt = 0; nt < 3; ++nt)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int row = mt * 8 + g, col = nt * 8 + 2 * t + i;
                if (nt < nb && row < N && col < N) X[row * N + col] = o[nt][i];
            }
        __syncwarp();
    }
    return res;
}

// A = D⁻¹ of an N x N block by pivoted Gauss-Jordan on one warp, in place:
// D is loaded into A's own storage and inverted there (the reference's pivot
// rule, first maximum |pivot| of each column, on the same column values as
// the augmented [D | I] form of rebuild_inverse; the row exchanges are undone
// as column exchanges at the end).  Lane l owns columns l + 32j for the
// row scaling and the elimination.  The pivot is found with the warp's
// integer max/min reductions on the bits of |x| (order-preserving for
// non-negative doubles; NaNs never win, ties go to the lowest row) and its
// value is broadcast from the lane that holds it, so no lane reads column k
// while its owner swaps rows; row k is scaled by one reciprocal.  `mult`
// (N doubles) and `perm` (N ints) are scratch.  Leaves log|det D| in
// misc[M_LOGDET] and flags a zero or nonfinite pivot in misc[M_ERR].
template <int S>
__device__ __forceinline__ void gj_invert_warp(double* A, double* mult, double* perm_area, int N, double* misc) {
    const int lane = threadIdx.x;
    int* perm = reinterpret_cast<int*>(perm_area);
    __syncwarp();
    double pivots[S];
#pragma unroll
    for (int j = 0; j < S; ++j) pivots[j] = 1.0;
    bool bad = false;
    for (int k = 0; k < N; ++k) {
        unsigned long long key = 0ull;
        int br = N;
        double bv = 0.0;
        for (int r = k + lane; r < N; r += 32) {
            const double x = A[r * N + k];
            const unsigned long long kx =
                isnan(x) ? 0ull : static_cast<unsigned long long>(__double_as_longlong(fabs(x))) + 1ull;
            if (kx > key) {
                key = kx;
                br = r;
                bv = x;
            }
        }
        const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
        const unsigned mhi = __reduce_max_sync(kAllLanes, hi);
        const unsigned mlo = __reduce_max_sync(kAllLanes, hi == mhi ? lo : 0u);
        const bool cand = hi == mhi && lo == mlo;
        const unsigned prow = __reduce_min_sync(kAllLanes, cand ? static_cast<unsigned>(br) : 0xffffffffu);
        const bool none = mhi == 0u && mlo == 0u;   // a column of NaNs has no pivot: flagged below
        const int piv = none ? k : static_cast<int>(prow);
        const unsigned owner = __ffs(__ballot_sync(kAllLanes, cand && br == piv && !none));
        double diag = __shfl_sync(kAllLanes, bv, owner ? owner - 1 : 0);
        if (none) diag = 0.0;
        bad |= diag == 0.0 || !isfinite(diag);
#pragma unroll
        for (int j = 0; j < S; ++j)
            if ((k >> 5) == j && lane == (k & 31)) pivots[j] = diag;
        const double inv = __drcp_rn(diag);
        // exchange rows k and piv; scale row k (its pivot entry becomes 1/diag)
        double pk[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const int c = lane + 32 * j;
            pk[j] = 0.0;
            if (c >= N) continue;
            const double xk = A[k * N + c], xp = A[piv * N + c];
            if (piv != k) A[piv * N + c] = xk;
            pk[j] = (c == k ? 1.0 : (piv != k ? xp : xk)) * inv;
            A[k * N + c] = pk[j];
        }
        if (lane == 0) perm[k] = piv;
        __syncwarp();
        // multipliers: column k of the other rows, which then starts from 0
        for (int r = lane; r < N; r += 32) {
            mult[r] = r == k ? 0.0 : A[r * N + k];
            if (r != k) A[r * N + k] = 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const int c = lane + 32 * j;
            if (c >= N) continue;
            for (int r0 = 0; r0 < N; r0 += 4) {
                double f[4], y[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = r0 + u;
                    const bool on = r < N && r != k;
                    f[u] = on ? mult[r] : 0.0;
                    y[u] = on ? A[r * N + c] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int r = r0 + u;
                    if (r < N && r != k) A[r * N + c] = y[u] - f[u] * pk[j];
                }
            }
        }
        __syncwarp();
    }
    // undo the row exchanges as column exchanges, last first
    for (int k = N - 1; k >= 0; --k) {
        const int pk = perm[k];
        if (pk != k)
            for (int r = lane; r < N; r += 32) {
                const double t = A[r * N + k];
                A[r * N + k] = A[r * N + pk];
                A[r * N + pk] = t;
            }
        __syncwarp();
    }
    double logdet = 0.0;
#pragma unroll
    for (int j = 0; j < S; ++j)
        if (lane + 32 * j < N) logdet += log(fabs(pivots[j]));
    logdet = warp_sum(logdet);
    if (lane == 0) {
        misc[M_LOGDET] = logdet;
        if (bad) misc[M_ERR] = 1.0;
    }
    __syncwarp();
}

// The same from the block's committed orbital rows D in the record: every
// column's loads first, then the inversion in A's storage.
template <int S>
__device__ __forceinline__ void gj_rebuild_warp(double* A, double* mult, double* perm_area, const double* D,
                                                int N, double* misc) {
    const int lane = threadIdx.x;
    __syncwarp();
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int c = lane + 32 * j;
        if (c >= N) continue;
        for (int r0 = 0; r0 < N; r0 += 8) {
            double t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t[u] = (r0 + u < N) ? __ldcg(D + (r0 + u) * N + c) : 0.0;
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (r0 + u < N) A[(r0 + u) * N + c] = t[u];
        }
    }
    gj_invert_warp<S>(A, mult, perm_area, N, misc);
}

// A = D⁻¹ of a twisted plane-wave block, D[r][c] = φ_c(x_r) recomputed from
// the positions (the particle `moved` at (mx, my)), by pivoted complex
// Gauss-Jordan on one warp in A's own storage (re plane Ar, im plane Ai,
// row-major, stride N).  The pivot of column k is the first row of largest
// |x|² at or below k, the rule of c_gj_rebuild; row k is scaled by
// (re, im) of 1/diag, the other rows lose their multiple of it, and the row
// exchanges are undone as column exchanges at the end.  Lane l owns columns
// l + 32j.  log|det D| accumulates pivot by pivot (0.5 ln|d|²) into
// misc[M_LOGDET]; a zero or nonfinite pivot is flagged in misc[M_ERR].
// `mult` (2N doubles) and `perm_area` (N ints) are scratch.
template <int S>
__device__ __noinline__ void cgj_rebuild_warp(const DevBlock& B, const double* pos, int moved, double mx, double my,
                                              double* Ar, double* Ai, double* mult, double* perm_area,
                                              double* misc) {
    const int lane = threadIdx.x, N = B.n;
    int* perm = reinterpret_cast<int*>(perm_area);
    __syncwarp();
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int c = lane + 32 * j;
        if (c >= N) continue;
        const double kx = B.k[c * 2], ky = B.k[c * 2 + 1];
        for (int r = 0; r < N; ++r) {
            const int part = B.first + r;
            const double x = part == moved ? mx : pos[part * 2];
            const double y = part == moved ? my : pos[part * 2 + 1];
            double sn, cs;
            sincos(fma(ky, y, kx * x), &sn, &cs);
            Ar[r * N + c] = cs;
            Ai[r * N + c] = sn;
        }
    }
    __syncwarp();
    double logdet = 0.0;
    bool bad = false;
    for (int k = 0; k < N; ++k) {
        double best = -1.0;
        int bi = N;
        for (int r = k + lane; r < N; r += 32) {
            const double xr = Ar[r * N + k], xi = Ai[r * N + k];
            const double a = xr * xr + xi * xi;
            if (a > best) {
                best = a;
                bi = r;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(kAllLanes, best, o);
            const int oi = __shfl_xor_sync(kAllLanes, bi, o);
            if (ob > best || (ob == best && oi < bi)) {
                best = ob;
                bi = oi;
            }
        }
        const int piv = bi >= N ? k : bi;   // a column of NaNs has no pivot: flagged
        bad |= !(best > 0.0) || !isfinite(best);
        logdet += 0.5 * log(best);
        const double dr = Ar[piv * N + k], di = Ai[piv * N + k];
        const double dd = dr * dr + di * di;
        const double ir = dr / dd, ii = -di / dd;
        __syncwarp();   // every lane has the pivot before rows move
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const int c = lane + 32 * j;
            if (c >= N) continue;
            double xr = Ar[piv * N + c], xi = Ai[piv * N + c];
            if (piv != k) {
                Ar[piv * N + c] = Ar[k * N + c];
                Ai[piv * N + c] = Ai[k * N + c];
            }
            if (c == k) {   // the inverse's column takes the place of column k
                xr = 1.0;
                xi = 0.0;
            }
            Ar[k * N + c] = xr * ir - xi * ii;
            Ai[k * N + c] = xr * ii + xi * ir;
        }
        if (lane == 0) perm[k] = piv;
        __syncwarp();
        for (int r = lane; r < N; r += 32) {
            mult[r] = r == k ? 0.0 : Ar[r * N + k];
            mult[N + r] = r == k ? 0.0 : Ai[r * N + k];
            if (r != k) Ar[r * N + k] = Ai[r * N + k] = 0.0;
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const int c = lane + 32 * j;
            if (c >= N) continue;
            const double qr = Ar[k * N + c], qi = Ai[k * N + c];
            for (int r = 0; r < N; ++r) {
                if (r == k) continue;
                const double fr = mult[r], fi = mult[N + r];
                Ar[r * N + c] -= fr * qr - fi * qi;
                Ai[r * N + c] -= fr * qi + fi * qr;
            }
        }
        __syncwarp();
    }
    for (int k = N - 1; k >= 0; --k) {
        const int pk = perm[k];
        if (pk != k)
            for (int r = lane; r < N; r += 32) {
                double t = Ar[r * N + k];
                Ar[r * N + k] = Ar[r * N + pk];
                Ar[r * N + pk] = t;
                t = Ai[r * N + k];
                Ai[r * N + k] = Ai[r * N + pk];
                Ai[r * N + pk] = t;
            }
        __syncwarp();
    }
    if (lane == 0) {
        misc[M_LOGDET] = logdet;
        if (bad) misc[M_ERR] = 1.0;
    }
    __syncwarp();
}

// Shared-memory view of the one-warp layout (DevSys f_*).  The sg, sl, kg,
// kl planes exist only in the local-energy phase (el = true), on top of the
// move scratch; `work` is the move union or the local energy's tables.
__device__ __forceinline__ Smem view_fast(const DevSys& s, double* sm, bool el) {
    Smem v{};
    v.pos = sm + s.f_pos;
    v.jg = sm + s.f_jg;
    v.jl = sm + s.f_jl;
    v.scal = sm + s.f_scal;
    v.rho = v.scal - s.o_scal + s.o_rho;
    v.nval = sm + s.f_nval;
    v.ngrad = sm + s.f_ngrad;
    v.nlap = sm + s.f_nlap;
    v.col = sm + s.f_col;
    v.rowp = sm + s.f_rowp;
    v.misc = sm + s.f_misc;
    v.cn = sm + s.f_cn;
    v.sn = sm + s.f_sn;
    v.co = sm + s.f_co;
    v.so = sm + s.f_so;
    v.work = sm + (el ? s.f_elwork : s.f_work);
    if (s.cplx) {   // phase planes of a complex ψ: in the hot part
        v.pg = v.scal - s.o_scal + s.o_pg;
        v.pl = v.scal - s.o_scal + s.o_pl;
    }
    if (el) {
        v.sg = sm + s.f_sg;
        v.sl = sm + s.f_sl;
        v.kg = sm + s.f_kg;
        v.kl = sm + s.f_kl;
    }
    return v;
}

// n doubles (n even, both ends 16-byte aligned) between a record (global,
// through L2 only: records stream through) and shared memory, by the warp.
__device__ __forceinline__ void copy_in_warp(double* dst, const double* src, int n) {
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    for (int i = threadIdx.x; i < n / 2; i += 32) d2[i] = __ldcg(s2 + i);
}

__device__ __forceinline__ void copy_out_warp(double* dst, const double* src, int n) {
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    for (int i = threadIdx.x; i < n / 2; i += 32) __stcg(d2 + i, s2[i]);
}

// The record's positions, pair-Jastrow planes and [scalars, end of the hot
// part) into the one-warp layout, and back.
__device__ __forceinline__ void load_fast(const DevSys& s, const double* rec, double* sm) {
    const int n2 = 2 * s.np;
    copy_in_warp(sm + s.f_pos, rec + s.o_pos, n2);
    copy_in_warp(sm + s.f_jg, rec + s.o_jg, n2);
    copy_in_warp(sm + s.f_jl, rec + s.o_jl, n2);
    copy_in_warp(sm + s.f_scal, rec + s.o_scal, s.hot - s.o_scal);
    __syncwarp();
}

__device__ __forceinline__ void store_fast(const DevSys& s, double* rec, const double* sm) {
    __syncwarp();
    const int n2 = 2 * s.np;
    copy_out_warp(rec + s.o_pos, sm + s.f_pos, n2);
    copy_out_warp(rec + s.o_jg, sm + s.f_jg, n2);
    copy_out_warp(rec + s.o_jl, sm + s.f_jl, n2);
    copy_out_warp(rec + s.o_scal, sm + s.f_scal, s.hot - s.o_scal);
    copy_out_warp(rec + s.o_sg, sm + s.f_sg, n2);
    copy_out_warp(rec + s.o_sl, sm + s.f_sl, n2);
    copy_out_warp(rec + s.o_kg, sm + s.f_kg, n2);
    copy_out_warp(rec + s.o_kl, sm + s.f_kl, n2);
}

// The local energy after a sweep: every particle's derivatives refreshed
// into the local-energy planes (zero for particles outside every determinant
// or image sum, as in the record), then kinetic + Ewald + open pair
// potentials.  Out of line: once per sweep.
template <int S>
__device__ __noinline__ double local_energy_warp(const DevSys& s, double* sm, const double* grec,
                                                 const int2* pairs, int npair) {
    const Smem v = view_fast(s, sm, true);
    __syncwarp();
    for (int i = threadIdx.x; i < 2 * s.np; i += 32) v.sg[i] = v.sl[i] = v.kg[i] = v.kl[i] = 0.0;
    __syncwarp();
    refresh_all<32, S>(s, v, grec);
    return local_energy<32, S>(s, v, pairs, npair);
}

// A pair term's u, u', u'' for the one-warp sweep: without zero-energy terms
// (ZE = false) only the inline Padé/Drummond forms are compiled, so the
// move's pair stage makes no function call.
template <bool ZE>
__device__ __forceinline__ void radial_w(const DevTerm& T, double r, double& u, double& du, double& d2u) {
    if constexpr (ZE)
        radial(T, r, u, du, d2u);
    else
        radial_pd(T, r, u, du, d2u);
}

// Select slot p >> 5 of a per-lane register array and read it from lane
// p & 31 (warp-uniform result).
template <int S, class T>
__device__ __forceinline__ T from_owner(const T (&x)[S], int p) {
    T mine = x[0];
#pragma unroll
    for (int j = 1; j < S; ++j)
        if ((p >> 5) == j) mine = x[j];
    return __shfl_sync(kAllLanes, mine, p & 31);
}

}  // namespace

}  // namespace alea_gpu
