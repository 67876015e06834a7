// Per-walker device functions of the sm_100a walker kernels: full evaluation,
// the pieces of a VMC/DMC sweep (propose → ratio → accept → commit for every
// particle, then the derivative refresh, E_L and the DMC branch factor).
//
// Algorithms restated from the reference (ItaloAlb/alea):
//   sweep          src/qmc/vmc.cpp:82-155 (Metropolis / Langevin),
//                  src/qmc/dmc.cpp:203-337 (Umrigar drift, node gate, drift
//                  Green's function), src/numerics/green_function.h:20-58
//   Slater         src/wavefunction/slater_determinant.cpp:395-437 (ratio),
//                  :515-726 (Sherman-Morrison commit and rebuild triggers),
//                  :862-903 (derivative refresh), :905-993 (Gauss-Jordan)
//   pair Jastrows  src/wavefunction/pade_jastrow.cpp:347-634,
//                  src/wavefunction/radial_pair_jastrow_impl.h
//   image sums     src/wavefunction/kspace_pair_sum.cpp:105-301
//   E_L            src/hamiltonian/kinetic.cpp:45-72, ewald_term.cpp:368-612,
//                  coulomb.cpp:31-61
//   branch weight  src/qmc/population_control.cpp:56-77
//   randoms        src/qmc/sweep_blocking.h:39-48
//
// Parallel layout: one CTA of NT threads per walker (NT = 32, 64 or 128,
// chosen per system: a move of a small system has only tens of independent
// items, and a one-warp CTA needs no cross-warp barrier).  Work inside a move
// is spread over orbitals (Slater), partners (pair terms), k-vectors (image
// sums) and matrix elements (rank-one update); partial sums meet in
// reductions.  Reciprocal phase ladders e^{inθ} are computed one entry per
// thread (sincos(nθ)) instead of by the serial recurrence.
//
// Deferred derivatives.  Like the reference's determinant (deferred partner
// refresh, slater_determinant.cpp:862-903), the k-space half of an image-summed
// Jastrow commits only ρ(k) and the moved particle's own derivatives; every
// other particle's k-space gradient and Laplacian is recomputed from ρ(k) and
// its phases when it is next read (its own move's drift, or the local energy).
// That turns the O(N·n_k) partner update of every accepted move into O(n_k)
// per read, and no per-particle phase cache is kept.
//
// This header holds the per-walker device functions (shared-memory view,
// Gauss-Jordan, complex and backflow determinants, refresh, ratio, commit,
// local energy, full evaluation); the kernels that use them live in
// alea_kernels.cu (generic CTA widths) and alea_fast.cu (the one-warp sweep).
#pragma once

#include <cstdio>

#include "alea_dev.cuh"
#include "alea_kernels.h"

namespace alea_gpu {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = 2.220446049250313e-16;
constexpr int kLad = 2 * (kMaxLadder + 1);   // doubles per ladder

struct Smem {
    double *pos, *jg, *jl, *kg, *kl, *sg, *sl, *scal, *rho, *pg, *pl;
    double *newpos, *nval, *ngrad, *nlap, *rad, *geo, *cn, *sn, *co, *so, *col, *rowp, *red,
        *misc, *lad, *work;
};

__device__ __forceinline__ Smem view(const DevSys& s, double* sm) {
    Smem v;
    v.pos = sm + s.o_pos;
    v.jg = sm + s.o_jg;
    v.jl = sm + s.o_jl;
    v.kg = sm + s.o_kg;
    v.kl = sm + s.o_kl;
    v.sg = sm + s.o_sg;
    v.sl = sm + s.o_sl;
    v.scal = sm + s.o_scal;
    v.rho = sm + s.o_rho;
    v.pg = sm + s.o_pg;
    v.pl = sm + s.o_pl;
    v.newpos = sm + s.s_newpos;
    v.nval = sm + s.s_nval;
    v.ngrad = sm + s.s_ngrad;
    v.nlap = sm + s.s_nlap;
    v.rad = sm + s.s_rad;
    v.geo = v.rad + static_cast<long>(s.np) * 4;
    v.cn = sm + s.s_cn;
    v.sn = sm + s.s_sn;
    v.co = sm + s.s_co;
    v.so = sm + s.s_so;
    v.col = sm + s.s_col;
    v.rowp = sm + s.s_rowp;
    v.red = sm + s.s_red;
    v.misc = sm + s.s_misc;
    v.lad = v.misc + 32;          // four ladders of kLad doubles
    v.work = sm + s.s_work;
    return v;
}

// misc slots
enum : int {
    M_R = 0, M_SCALE, M_LOGR, M_PHASE, M_ACCEPT, M_REBUILD, M_LOGDET, M_ERR, M_U, M_SCFWD,
    M_GOX, M_GOY, M_SGX, M_SGY, M_SLX, M_SLY, M_JGX, M_JGY, M_JLX, M_JLY, M_KGX, M_KGY,
    M_KLX, M_KLY, M_RI /* Im R */, M_PGX, M_PGY, M_PLX, M_PLY /* phase part at the proposal */,
    M_LOGDR /* determinant part of the log ratio */
};

template <int NT>
__device__ __forceinline__ void load_hot(const DevSys& s, const double* rec, double* sm) {
    const double2* src = reinterpret_cast<const double2*>(rec);
    double2* dst = reinterpret_cast<double2*>(sm);
    for (int i = threadIdx.x; i < s.hot / 2; i += NT) dst[i] = src[i];
    __syncthreads();
}

template <int NT>
__device__ __forceinline__ void store_hot(const DevSys& s, double* rec, const double* sm) {
    __syncthreads();
    const double2* src = reinterpret_cast<const double2*>(sm);
    double2* dst = reinterpret_cast<double2*>(rec);
    for (int i = threadIdx.x; i < s.hot / 2; i += NT) dst[i] = src[i];
}

__device__ __forceinline__ int block_of(const DevSys& s, int p) {
    for (int b = 0; b < s.nblocks; ++b)
        if (p >= s.blocks[b].first && p < s.blocks[b].last) return b;
    return -1;
}

__device__ __forceinline__ bool kspace_of(const DevSys& s, int p) {
    for (int t = 0; t < s.nterms; ++t)
        if (s.terms[t].image && in_term(s.terms[t], p)) return true;
    return false;
}

// Ladders e^{inθ_q}, n = 0..m_q, of up to four angles, one entry per thread,
// into out[q*kLad + 2n], out[q*kLad + 2n + 1].  No barrier.
template <int NT>
__device__ __forceinline__ void ladders(const double* theta, const int* m, int nq, double* out) {
    int total = 0;
    for (int q = 0; q < nq; ++q) total += m[q] + 1;
    for (int e = threadIdx.x; e < total; e += NT) {
        int q = 0, n = e;
        while (n > m[q]) {
            n -= m[q] + 1;
            ++q;
        }
        double c, sn;
        if (n == 0) {
            c = 1.0;
            sn = 0.0;
        } else {
            sincos(static_cast<double>(n) * theta[q], &sn, &c);
        }
        out[q * kLad + 2 * n] = c;
        out[q * kLad + 2 * n + 1] = sn;
    }
}

__device__ __forceinline__ void ladder_pick(const double* lad, int n, double& re, double& im) {
    const int a = n < 0 ? -n : n;
    re = lad[2 * a];
    im = n < 0 ? -lad[2 * a + 1] : lad[2 * a + 1];
}

// e^{ik·r} for the Jastrow k set from the two ladders of r.
__device__ __forceinline__ void phase_k(const DevSys& s, const double* l1, const double* l2, int k,
                                        double& c, double& sn) {
    double ar, ai, br, bi;
    ladder_pick(l1, s.n1J[k], ar, ai);
    ladder_pick(l2, s.n2J[k], br, bi);
    c = ar * br - ai * bi;
    sn = ar * bi + ai * br;
}

// Gradient/Laplacian terms of one k for a particle with phases (c, sn) that
// sees the density (pr, pi) (kspace_pair_sum.cpp:76-97).
__device__ __forceinline__ void kterm(const DevSys& s, double w, int k, double c, double sn,
                                      double pr, double pi, double self, double* acc) {
    const double g = 2.0 * w * (c * pi - sn * pr);
    const double l = 2.0 * w * (self - (c * pr + sn * pi));
    acc[0] += s.kxJ[k] * g;
    acc[1] += s.kyJ[k] * g;
    acc[2] += s.kx2J[k] * l;
    acc[3] += s.ky2J[k] * l;
}

// Every image-summed term's k-space gradient/Laplacian of particle i (group
// gi) from its phases, added to acc[4].
__device__ __forceinline__ void kspace_particle_k(const DevSys& s, const Smem& v, int i, int gi, int k,
                                                  double c, double sn, double* acc) {
    const int nk = s.nkJ;
    for (int t = 0; t < s.nterms; ++t) {
        const DevTerm& T = s.terms[t];
        if (!T.image || !in_term(T, i)) continue;
        const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
        const int go = T.same0 ? gi : (gi == ga ? gb : ga);
        const double* pr = v.rho + go * 2 * nk;
        kterm(s, T.kw[k], k, c, sn, pr[k], pr[nk + k], T.same0 ? 1.0 : 0.0, acc);
    }
}

// Visit the elements (r, c) of an N×N matrix with the CTA's NT threads, no
// integer division inside the loop: when N ≤ NT each thread owns column c and
// rows r0, r0 + NT/N, ... (⌊NT/N⌋ rows in flight); otherwise each thread owns
// columns c, c + NT, ... and walks all rows.
template <int NT, class F>
__device__ __forceinline__ void for_each_elem(int N, F&& f) {
    if (N <= NT) {
        const int per = NT / N;
        if (static_cast<int>(threadIdx.x) < per * N) {
            const int r0 = static_cast<int>(threadIdx.x) / N;
            const int c = static_cast<int>(threadIdx.x) - r0 * N;
            for (int r = r0; r < N; r += per) f(r, c);
        }
    } else {
        for (int c = threadIdx.x; c < N; c += NT)
            for (int r = 0; r < N; ++r) f(r, c);
    }
}

// ───────────────────────── Gauss-Jordan rebuild ─────────────────────────

// A = D⁻¹ of block b from its committed rows in HBM, by pivoted Gauss-Jordan
// (first maximum |pivot| in each column, as the reference's rebuild_inverse).
// Leaves log|det D| in misc[M_LOGDET]; flags a singular matrix in misc[M_ERR].
template <int NT>
__device__ void gj_rebuild(const DevSys& s, const Smem& v, const double* grec, int b) {
    const DevBlock& B = s.blocks[b];
    const int N = B.n;
    double* A = v.scal - s.o_scal + B.oA;
    double* m = v.work;
    const double* D = grec + B.oD;
    __syncthreads();
    for_each_elem<NT>(N, [&](int r, int c) {
        m[r * N + c] = D[r * N + c];
        A[r * N + c] = (r == c) ? 1.0 : 0.0;
    });
    if (threadIdx.x == 0) v.misc[M_LOGDET] = 0.0;
    __syncthreads();
    __shared__ int s_piv;
    for (int k = 0; k < N; ++k) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = N;
            for (int r = k + static_cast<int>(threadIdx.x); r < N; r += 32) {
                const double a = fabs(m[r * N + k]);
                if (a > best) {
                    best = a;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                if (bi >= N) bi = k;   // a column of NaNs has no pivot: flagged below
                s_piv = bi;
                const double diag = m[bi * N + k];
                if (diag == 0.0 || !isfinite(diag)) v.misc[M_ERR] = 1.0;
                v.misc[M_LOGDET] += log(fabs(diag));
            }
        }
        __syncthreads();
        const int piv = s_piv;
        if (piv != k)
            for (int c = threadIdx.x; c < N; c += NT) {
                double t = m[k * N + c];
                m[k * N + c] = m[piv * N + c];
                m[piv * N + c] = t;
                t = A[k * N + c];
                A[k * N + c] = A[piv * N + c];
                A[piv * N + c] = t;
            }
        __syncthreads();
        const double diag = m[k * N + k];
        __syncthreads();
        for (int c = threadIdx.x; c < N; c += NT) {
            m[k * N + c] /= diag;
            A[k * N + c] /= diag;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < N; r += NT) v.col[r] = m[r * N + k];
        __syncthreads();
        for_each_elem<NT>(N, [&](int r, int c) {
            if (r == k) return;
            const double f = v.col[r];
            m[r * N + c] -= f * m[k * N + c];
            A[r * N + c] -= f * A[k * N + c];
        });
        __syncthreads();
    }
}

// ───────────────────────── complex determinant ─────────────────────────
//
// Twisted plane waves φ_m = e^{i q_m·r} (complex_orbital_set.h:78-182) in a
// complex determinant (complex_slater_determinant.cpp).  The inverse lives in
// shared memory as re[N²] then im[N²]; the orbital rows are recomputed from
// the positions when needed (one sincos each), so nothing is kept in HBM.
// With t = A[m][kr] φ_m(r): ∂_d φ = i q_d φ and ∂²_d φ = -q_d² φ give
// G_d = Σ_m i q_d t and Lraw_d = Σ_m -q_d² t.

__device__ __forceinline__ void c_orb(const DevBlock& B, int m, const double* r, double& c, double& sn) {
    const double arg = fma(B.k[m * 2 + 1], r[1], B.k[m * 2] * r[0]);
    sincos(arg, &sn, &c);
}

// One orbital's contributions at r to R = Σ t, G and Lraw (re and im).
__device__ __forceinline__ void c_accumulate(const DevBlock& B, int m, double ar, double ai, double c,
                                             double sn, double* R, double* Gr, double* Gi,
                                             double* Lr, double* Li) {
    const double tr = ar * c - ai * sn, ti = ar * sn + ai * c;
    R[0] += tr;
    R[1] += ti;
    for (int d = 0; d < 2; ++d) {
        const double q = B.k[m * 2 + d];
        Gr[d] += -q * ti;
        Gi[d] += q * tr;
        Lr[d] += -q * q * tr;
        Li[d] += -q * q * ti;
    }
}

// A = D⁻¹ of block b, D[kr][m] = φ_m(r_kr) (particle `moved` at `npos`), by
// Gauss-Jordan with the pivot of largest modulus.  log|det D| to
// misc[M_LOGDET], a singular matrix flagged in misc[M_ERR].
template <int NT>
__device__ void c_gj_rebuild(const DevSys& s, const Smem& v, int b, int moved, const double* npos) {
    const DevBlock& B = s.blocks[b];
    const int N = B.n, NN = N * N;
    double* Ar = v.scal - s.o_scal + B.oA;
    double* Ai = Ar + ((NN + 3) & ~3);
    double* mr = v.work;
    double* mi = v.work + NN;
    __syncthreads();
    for_each_elem<NT>(N, [&](int r, int c) {
        const int part = B.first + r;
        const double* pr = part == moved ? npos : v.pos + part * 2;
        double cs, sn;
        c_orb(B, c, pr, cs, sn);
        mr[r * N + c] = cs;
        mi[r * N + c] = sn;
        Ar[r * N + c] = (r == c) ? 1.0 : 0.0;
        Ai[r * N + c] = 0.0;
    });
    if (threadIdx.x == 0) v.misc[M_LOGDET] = 0.0;
    __syncthreads();
    __shared__ int s_piv;
    for (int k = 0; k < N; ++k) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = N;
            for (int r = k + static_cast<int>(threadIdx.x); r < N; r += 32) {
                const double a = mr[r * N + k] * mr[r * N + k] + mi[r * N + k] * mi[r * N + k];
                if (a > best) {
                    best = a;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                if (bi >= N) bi = k;   // a column of NaNs has no pivot: flagged below
                s_piv = bi;
                if (!(best > 0.0) || !isfinite(best)) v.misc[M_ERR] = 1.0;
                v.misc[M_LOGDET] += 0.5 * log(best);
            }
        }
        __syncthreads();
        const int piv = s_piv;
        if (piv != k)
            for (int c = threadIdx.x; c < N; c += NT) {
                double t = mr[k * N + c]; mr[k * N + c] = mr[piv * N + c]; mr[piv * N + c] = t;
                t = mi[k * N + c]; mi[k * N + c] = mi[piv * N + c]; mi[piv * N + c] = t;
                t = Ar[k * N + c]; Ar[k * N + c] = Ar[piv * N + c]; Ar[piv * N + c] = t;
                t = Ai[k * N + c]; Ai[k * N + c] = Ai[piv * N + c]; Ai[piv * N + c] = t;
            }
        __syncthreads();
        const double dr = mr[k * N + k], di = mi[k * N + k];
        const double dd = dr * dr + di * di;
        const double ir = dr / dd, ii = -di / dd;   // 1 / diag
        __syncthreads();
        for (int c = threadIdx.x; c < N; c += NT) {
            double xr = mr[k * N + c], xi = mi[k * N + c];
            mr[k * N + c] = xr * ir - xi * ii;
            mi[k * N + c] = xr * ii + xi * ir;
            xr = Ar[k * N + c];
            xi = Ai[k * N + c];
            Ar[k * N + c] = xr * ir - xi * ii;
            Ai[k * N + c] = xr * ii + xi * ir;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < N; r += NT) {
            v.col[r] = mr[r * N + k];
            v.col[N + r] = mi[r * N + k];
        }
        __syncthreads();
        for_each_elem<NT>(N, [&](int r, int c) {
            if (r == k) return;
            const double fr = v.col[r], fi = v.col[N + r];
            const double pr_ = mr[k * N + c], pi_ = mi[k * N + c];
            mr[r * N + c] -= fr * pr_ - fi * pi_;
            mi[r * N + c] -= fr * pi_ + fi * pr_;
            const double qr = Ar[k * N + c], qi = Ai[k * N + c];
            Ar[r * N + c] -= fr * qr - fi * qi;
            Ai[r * N + c] -= fr * qi + fi * qr;
        });
        __syncthreads();
    }
}

// Modulus and phase parts of ∇ln ψ and ∂²ln ψ of the complex determinant for
// every particle of every block, one particle per thread.
template <int NT>
__device__ void c_refresh_all(const DevSys& s, const Smem& v) {
    for (int b = 0; b < s.nblocks; ++b) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n;
        const double* Ar = v.scal - s.o_scal + B.oA;
        const double* Ai = Ar + ((N * N + 3) & ~3);
        for (int kr = threadIdx.x; kr < N; kr += NT) {
            const int part = B.first + kr;
            double R[2] = {0, 0}, Gr[2] = {0, 0}, Gi[2] = {0, 0}, Lr[2] = {0, 0}, Li[2] = {0, 0};
            for (int m = 0; m < N; ++m) {
                double cs, sn;
                c_orb(B, m, v.pos + part * 2, cs, sn);
                c_accumulate(B, m, Ar[m * N + kr], Ai[m * N + kr], cs, sn, R, Gr, Gi, Lr, Li);
            }
            for (int d = 0; d < 2; ++d) {
                v.sg[part * 2 + d] = Gr[d];
                v.pg[part * 2 + d] = Gi[d];
                v.sl[part * 2 + d] = Lr[d] - (Gr[d] * Gr[d] - Gi[d] * Gi[d]);
                v.pl[part * 2 + d] = Li[d] - 2.0 * Gr[d] * Gi[d];
            }
        }
    }
    __syncthreads();
}

// ───────────────────────── backflow determinant ───────────────────────
//
// BackflowSlaterDeterminant (backflow_slater_determinant.cpp,
// backflow_transformation.cpp): M[i][m] = φ_m(x_i) with quasi-coordinates
// x_i = r_i + Σ_c Σ_j η_c(r_ij) r_ij, η = (1 - r/L)^C Σ_k c_k r^k.  A move of
// p shifts every row it displaces and rebuilds p's own row; the new matrix
// is inverted by pivoted Gauss-Jordan (no rank-one update applies), which
// gives the ratio of determinants and, with F = Aᵀ∇φ(x) and the pair
// tensors B(r) = η δ + η' r̂ r̂ᵀ r, the moved particle's gradient.  The
// determinant part of every particle's ∇ and ∂² ln ψ lives in sg/sl (a
// backflow system has no plain blocks), refreshed before it is read.

__device__ __forceinline__ void bf_eta(const DevBFCh& C, double r, double& eta, double& e1, double& e2) {
    if (r >= C.L) {
        eta = e1 = e2 = 0.0;
        return;
    }
    const double t = 1.0 - r / C.L;
    double tc2 = 1.0;
    for (int i = 0; i < C.C - 2; ++i) tc2 *= t;
    const double f = tc2 * t * t;
    const double fp = -static_cast<double>(C.C) / C.L * tc2 * t;
    const double fpp = static_cast<double>(C.C) * static_cast<double>(C.C - 1) / (C.L * C.L) * tc2;
    double P = 0.0, Pp = 0.0, Ppp = 0.0;
    for (int k = C.nc - 1; k >= 0; --k) {
        Ppp = Ppp * r + 2.0 * Pp;
        Pp = Pp * r + P;
        P = P * r + C.c[k];
    }
    eta = f * P;
    e1 = fp * P + f * Pp;
    e2 = fpp * P + 2.0 * fp * Pp + f * Ppp;
}

// One pair r_ij = ri - rj (minimum image): adds sign·η r_ij to x; fills the
// tensors B and S (2x2, row α, column β) when B is given.  False beyond L.
__device__ __forceinline__ bool bf_pair(const DevSys& s, const DevBFCh& C, const double* ri, const double* rj,
                                        double sign, double* x, double* B, double* S) {
    double del[3] = {ri[0] - rj[0], ri[1] - rj[1], 0.0};
    min_image(s, del);
    const double r = sqrt(del[0] * del[0] + del[1] * del[1]);
    if (r >= C.L) return false;
    double eta, e1, e2;
    bf_eta(C, r, eta, e1, e2);
    x[0] += sign * eta * del[0];
    x[1] += sign * eta * del[1];
    if (B) {
        const double inv_r = r > 0.0 ? 1.0 / r : 0.0;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                B[a * 2 + b] = (a == b ? eta : 0.0) + e1 * del[a] * del[b] * inv_r;
                const double rb2 = del[b] * del[b] * inv_r * inv_r;
                S[a * 2 + b] = (a == b ? 2.0 * e1 * del[b] * inv_r : 0.0) +
                               del[a] * (e2 * rb2 + e1 * inv_r * (1.0 - rb2));
            }
    }
    return true;
}

__device__ __forceinline__ bool bf_affects(const DevBF& D, int k) {
    if (k >= D.first && k < D.last) return true;
    for (int c = 0; c < D.nch; ++c)
        if (k >= D.ch[c].sf && k < D.ch[c].sl) return true;
    return false;
}

// Orbital m at x: value, gradient, Hessian [a*2+b].
__device__ __forceinline__ void bf_orbital(const DevSys& s, const DevBF& D, int m, const double* x, double& val,
                                           double* g, double* h) {
    if (D.type == 0) {
        const double kx = D.k[m * 2], ky = D.k[m * 2 + 1];
        double sn, c;
        sincos(kx * x[0] + ky * x[1], &sn, &c);
        const bool is_s = D.is_sin[m] != 0.0;
        const double v = is_s ? sn : c, dv = is_s ? c : -sn;
        val = v;
        g[0] = kx * dv;
        g[1] = ky * dv;
        if (h) {
            h[0] = -kx * kx * v;
            h[1] = h[2] = -kx * ky * v;
            h[3] = -ky * ky * v;
        }
    } else {
        const double al = D.alphas[m];
        double del[3] = {x[0] - D.centers[m * 2], x[1] - D.centers[m * 2 + 1], 0.0};
        min_image(s, del);
        const double phi = exp(-al * (del[0] * del[0] + del[1] * del[1]));
        val = phi;
        g[0] = -2.0 * al * del[0] * phi;
        g[1] = -2.0 * al * del[1] * phi;
        if (h) {
            h[0] = (4.0 * al * al * del[0] * del[0] - 2.0 * al) * phi;
            h[1] = h[2] = 4.0 * al * al * del[0] * del[1] * phi;
            h[3] = (4.0 * al * al * del[1] * del[1] - 2.0 * al) * phi;
        }
    }
}

// Pivoted Gauss-Jordan of m (N×N, destroyed) into a, with log|det| and sign
// to out[0], out[1] and out[2] = 1 when regular (pivot of largest modulus,
// ties to the lowest row).
template <int NT>
__device__ void bf_invert(int N, double* m, double* a, double* col, double* out) {
    __syncthreads();
    for_each_elem<NT>(N, [&](int r, int c) { a[r * N + c] = (r == c) ? 1.0 : 0.0; });
    if (threadIdx.x == 0) {
        out[0] = 0.0;
        out[1] = 1.0;
        out[2] = 1.0;
    }
    __syncthreads();
    __shared__ int s_piv;
    for (int k = 0; k < N; ++k) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = N;
            for (int r = k + static_cast<int>(threadIdx.x); r < N; r += 32) {
                const double v = fabs(m[r * N + k]);
                if (v > best) {
                    best = v;
                    bi = r;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (threadIdx.x == 0) {
                if (bi >= N) bi = k;   // a column of NaNs has no pivot: flagged below
                s_piv = bi;
                const double diag = m[bi * N + k];
                if (diag == 0.0 || !isfinite(diag)) {
                    out[2] = 0.0;
                } else {
                    out[0] += log(fabs(diag));
                    if (diag < 0.0) out[1] = -out[1];
                    if (bi != k) out[1] = -out[1];
                }
            }
        }
        __syncthreads();
        if (out[2] == 0.0) return;
        const int piv = s_piv;
        if (piv != k)
            for (int c = threadIdx.x; c < N; c += NT) {
                double t = m[k * N + c]; m[k * N + c] = m[piv * N + c]; m[piv * N + c] = t;
                t = a[k * N + c]; a[k * N + c] = a[piv * N + c]; a[piv * N + c] = t;
            }
        __syncthreads();
        const double inv = 1.0 / m[k * N + k];
        __syncthreads();
        for (int c = threadIdx.x; c < N; c += NT) {
            m[k * N + c] *= inv;
            a[k * N + c] *= inv;
        }
        __syncthreads();
        for (int r = threadIdx.x; r < N; r += NT) col[r] = m[r * N + k];
        __syncthreads();
        for_each_elem<NT>(N, [&](int r, int c) {
            if (r == k) return;
            const double f = col[r];
            m[r * N + c] -= f * m[k * N + c];
            a[r * N + c] -= f * a[k * N + c];
        });
        __syncthreads();
    }
}

// x_t from scratch: r_t + Σ_c Σ_j η(r_tj) r_tj, with particle `moved` at npos.
__device__ __forceinline__ void bf_row_x(const DevSys& s, const DevBF& D, const double* pos, int moved,
                                         const double* npos, int P, double* xt) {
    const double* rp = P == moved ? npos : pos + P * 2;
    xt[0] = rp[0];
    xt[1] = rp[1];
    for (int c = 0; c < D.nch; ++c)
        for (int j = D.ch[c].sf; j < D.ch[c].sl; ++j) {
            if (j == P) continue;
            const double* rj = j == moved ? npos : pos + j * 2;
            bf_pair(s, D.ch[c], rp, rj, 1.0, xt, nullptr, nullptr);
        }
}

// ∂_k ln|D| = F_k (1 + Σ_j B(r_kj)) - Σ_t F_t B(r_tk) at the given positions,
// summed over the CTA (all threads return it).
template <int NT>
__device__ void bf_grad_of(const DevSys& s, const Smem& v, const DevBF& D, const double* F, int k, int moved,
                           const double* npos, double* g) {
    const int N = D.n, np = s.np;
    const double* rk = k == moved ? npos : v.pos + k * 2;
    const int tk = (k >= D.first && k < D.last) ? k - D.first : -1;
    double acc[2] = {0.0, 0.0};
    // own row: F_k e_β and F_k·B(r_kj) over the sources
    if (tk >= 0) {
        const double* Fk = F + tk * 2;
        if (threadIdx.x == 0) {
            acc[0] += Fk[0];
            acc[1] += Fk[1];
        }
        for (int j = threadIdx.x; j < np; j += NT) {
            if (j == k) continue;
            const double* rj = j == moved ? npos : v.pos + j * 2;
            for (int c = 0; c < D.nch; ++c) {
                if (j < D.ch[c].sf || j >= D.ch[c].sl) continue;
                double unused[2] = {0, 0}, B[4], S[4];
                if (!bf_pair(s, D.ch[c], rk, rj, 1.0, unused, B, S)) continue;
                for (int a = 0; a < 2; ++a)
                    for (int b = 0; b < 2; ++b) acc[b] += Fk[a] * B[a * 2 + b];
            }
        }
    }
    // the rows that k displaces: - F_t·B(r_tk)
    for (int t = threadIdx.x; t < N; t += NT) {
        const int P = D.first + t;
        if (P == k) continue;
        const double* rt = P == moved ? npos : v.pos + P * 2;
        for (int c = 0; c < D.nch; ++c) {
            if (k < D.ch[c].sf || k >= D.ch[c].sl) continue;
            double unused[2] = {0, 0}, B[4], S[4];
            if (!bf_pair(s, D.ch[c], rt, rk, 1.0, unused, B, S)) continue;
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) acc[b] -= F[t * 2 + a] * B[a * 2 + b];
        }
    }
    block_sum<NT>(acc, v.red);
    g[0] = acc[0];
    g[1] = acc[1];
}

// The proposal of p for determinant d: pending x', A', F', (log|det|', sign'),
// p's gradient and validity in the pending area.
template <int NT>
__device__ void bf_propose(const DevSys& s, const Smem& v, int d, int p) {
    const DevBF& D = s.bf[d];
    const int N = D.n;
    double* sm = v.scal - s.o_scal;   // shared-memory base
    const double* x = sm + D.oX;
    double* px = sm + D.pX;
    double* pa = sm + D.pA;
    double* pf = sm + D.pF;
    double* pm = sm + D.pM;
    // x': shift the rows p displaces, rebuild p's own row
    for (int t = threadIdx.x; t < N; t += NT) {
        const int P = D.first + t;
        if (P == p) {
            bf_row_x(s, D, v.pos, p, v.newpos, P, px + t * 2);
            continue;
        }
        double xt[2] = {x[t * 2], x[t * 2 + 1]};
        for (int c = 0; c < D.nch; ++c) {
            if (p < D.ch[c].sf || p >= D.ch[c].sl) continue;
            bf_pair(s, D.ch[c], v.pos + P * 2, v.newpos, 1.0, xt, nullptr, nullptr);
            bf_pair(s, D.ch[c], v.pos + P * 2, v.pos + p * 2, -1.0, xt, nullptr, nullptr);
        }
        px[t * 2] = xt[0];
        px[t * 2 + 1] = xt[1];
    }
    __syncthreads();
    double* mrows = v.work;
    for_each_elem<NT>(N, [&](int i, int m) {
        double val, g[2];
        bf_orbital(s, D, m, px + i * 2, val, g, nullptr);
        mrows[i * N + m] = val;
    });
    bf_invert<NT>(N, mrows, pa, v.col, pm);
    if (pm[2] == 0.0) {
        __syncthreads();
        return;
    }
    // F'_i = Σ_m A'[m][i] ∇φ_m(x'_i)
    for (int i = threadIdx.x; i < N; i += NT) {
        double f0 = 0.0, f1 = 0.0;
        for (int m = 0; m < N; ++m) {
            double val, g[2];
            bf_orbital(s, D, m, px + i * 2, val, g, nullptr);
            const double a = pa[m * N + i];
            f0 += a * g[0];
            f1 += a * g[1];
        }
        pf[i * 2] = f0;
        pf[i * 2 + 1] = f1;
    }
    __syncthreads();
    double g[2];
    bf_grad_of<NT>(s, v, D, pf, p, p, v.newpos, g);
    if (threadIdx.x == 0) {
        pm[3] = g[0];
        pm[4] = g[1];
    }
    __syncthreads();
}

// Every particle's determinant gradient and Laplacian of backflow
// determinant d from the committed A and F, with x rebuilt from the
// positions (BackflowSlaterDeterminant::refresh_walker); added into
// sg/sl (zeroed by the caller).  evaluate != 0: the matrix is inverted and F
// formed first (a full evaluation).
template <int NT>
__device__ void bf_derivatives(const DevSys& s, const Smem& v, int d, bool evaluate) {
    const DevBF& D = s.bf[d];
    const int N = D.n, np = s.np;
    double* sm = v.scal - s.o_scal;
    double* x = sm + D.oX;
    double* A = sm + D.oA;
    double* F = sm + D.oF;
    double* ls = sm + D.oLS;
    for (int t = threadIdx.x; t < N; t += NT) bf_row_x(s, D, v.pos, -1, nullptr, D.first + t, x + t * 2);
    __syncthreads();
    double* grow = v.work;                 // ∇φ_m(x_r) [(r*N + m)*2 + α]
    double* G = v.work + 2 * N * N;        // G^α[j][r] at [α*N*N + j*N + r]
    double* T = G + 2 * N * N;             // T_i [i*4 + αγ]
    double* V = T + 4 * N;                 // Jacobian columns [β][t*2 + α]
    if (evaluate) {
        for_each_elem<NT>(N, [&](int i, int m) {
            double val, g[2];
            bf_orbital(s, D, m, x + i * 2, val, g, nullptr);
            grow[i * N + m] = val;
        });
        bf_invert<NT>(N, grow, A, v.col, v.misc + M_U);   // misc[M_U..M_U+2] scratch
        if (threadIdx.x == 0) {
            ls[0] = v.misc[M_U];
            ls[1] = v.misc[M_U + 1];
            if (v.misc[M_U + 2] == 0.0) v.scal[S_ERR] = 1.0;
        }
        __syncthreads();
    }
    for_each_elem<NT>(N, [&](int r, int m) {
        double val, g[2];
        bf_orbital(s, D, m, x + r * 2, val, g, nullptr);
        grow[(r * N + m) * 2] = g[0];
        grow[(r * N + m) * 2 + 1] = g[1];
    });
    __syncthreads();
    if (evaluate) {
        for (int i = threadIdx.x; i < N; i += NT) {
            double f0 = 0.0, f1 = 0.0;
            for (int m = 0; m < N; ++m) {
                f0 += A[m * N + i] * grow[(i * N + m) * 2];
                f1 += A[m * N + i] * grow[(i * N + m) * 2 + 1];
            }
            F[i * 2] = f0;
            F[i * 2 + 1] = f1;
        }
    }
    for (int i = threadIdx.x; i < N; i += NT) {
        double t4[4] = {0, 0, 0, 0};
        for (int m = 0; m < N; ++m) {
            double val, g[2], h[4];
            bf_orbital(s, D, m, x + i * 2, val, g, h);
            for (int q = 0; q < 4; ++q) t4[q] += A[m * N + i] * h[q];
        }
        for (int q = 0; q < 4; ++q) T[i * 4 + q] = t4[q];
    }
    for_each_elem<NT>(N, [&](int j, int r) {
        double g0 = 0.0, g1 = 0.0;
        for (int m = 0; m < N; ++m) {
            g0 += A[m * N + j] * grow[(r * N + m) * 2];
            g1 += A[m * N + j] * grow[(r * N + m) * 2 + 1];
        }
        G[j * N + r] = g0;
        G[N * N + j * N + r] = g1;
    });
    __syncthreads();
    for (int k = 0; k < np; ++k) {
        if (!bf_affects(D, k)) continue;
        const int tk = (k >= D.first && k < D.last) ? k - D.first : -1;
        // Jacobian columns v_β (β = 0, 1) over the rows, and Σ F·S
        double fs[2] = {0.0, 0.0};
        for (int t = threadIdx.x; t < N; t += NT) {
            double vt[2][2] = {{0, 0}, {0, 0}};
            const int P = D.first + t;
            if (t == tk) {
                vt[0][0] = 1.0;
                vt[1][1] = 1.0;
                for (int c = 0; c < D.nch; ++c)
                    for (int j = D.ch[c].sf; j < D.ch[c].sl; ++j) {
                        if (j == k) continue;
                        double unused[2] = {0, 0}, B[4], S[4];
                        if (!bf_pair(s, D.ch[c], v.pos + k * 2, v.pos + j * 2, 1.0, unused, B, S)) continue;
                        for (int be = 0; be < 2; ++be)
                            for (int a = 0; a < 2; ++a) {
                                vt[be][a] += B[a * 2 + be];
                                fs[be] += F[t * 2 + a] * S[a * 2 + be];
                            }
                    }
            } else {
                for (int c = 0; c < D.nch; ++c) {
                    if (k < D.ch[c].sf || k >= D.ch[c].sl) continue;
                    double unused[2] = {0, 0}, B[4], S[4];
                    if (!bf_pair(s, D.ch[c], v.pos + P * 2, v.pos + k * 2, 1.0, unused, B, S)) continue;
                    for (int be = 0; be < 2; ++be)
                        for (int a = 0; a < 2; ++a) {
                            vt[be][a] = -B[a * 2 + be];
                            fs[be] += F[t * 2 + a] * S[a * 2 + be];
                        }
                }
            }
            for (int be = 0; be < 2; ++be) {
                V[be * 2 * N + t * 2] = vt[be][0];
                V[be * 2 * N + t * 2 + 1] = vt[be][1];
            }
        }
        __syncthreads();
        // Σ_t vᵀ T_t v and - Σ_{j,r} U_jr U_rj, U_jr = Σ_α v_rα G^α[j][r]
        double acc[4] = {fs[0], fs[1], 0.0, 0.0};
        for (int t = threadIdx.x; t < N; t += NT)
            for (int be = 0; be < 2; ++be) {
                const double* vt = V + be * 2 * N + t * 2;
                const double* Tt = T + t * 4;
                acc[be] += vt[0] * vt[0] * Tt[0] + vt[0] * vt[1] * (Tt[1] + Tt[2]) + vt[1] * vt[1] * Tt[3];
            }
        for_each_elem<NT>(N, [&](int j, int r) {
            for (int be = 0; be < 2; ++be) {
                const double* Vb = V + be * 2 * N;
                const double ujr = Vb[r * 2] * G[j * N + r] + Vb[r * 2 + 1] * G[N * N + j * N + r];
                const double urj = Vb[j * 2] * G[r * N + j] + Vb[j * 2 + 1] * G[N * N + r * N + j];
                acc[be] -= ujr * urj;
            }
        });
        block_sum<NT>(acc, v.red);
        double g[2];
        bf_grad_of<NT>(s, v, D, F, k, -1, nullptr, g);
        if (threadIdx.x == 0) {
            v.sg[k * 2] += g[0];
            v.sg[k * 2 + 1] += g[1];
            v.sl[k * 2] += acc[0];
            v.sl[k * 2 + 1] += acc[1];
        }
        __syncthreads();
    }
}

// Every backflow determinant's contribution to every particle (sg, sl).
template <int NT>
__device__ void bf_refresh_all(const DevSys& s, const Smem& v, bool evaluate) {
    for (int i = threadIdx.x; i < s.np * 2; i += NT) v.sg[i] = v.sl[i] = 0.0;
    __syncthreads();
    for (int d = 0; d < s.nbf; ++d) bf_derivatives<NT>(s, v, d, evaluate);
}

// The drift's refresh of p: its determinant gradient from the committed F.
template <int NT>
__device__ void bf_refresh_particle(const DevSys& s, const Smem& v, int p) {
    double tot[2] = {0.0, 0.0};
    for (int d = 0; d < s.nbf; ++d) {
        const DevBF& D = s.bf[d];
        if (!bf_affects(D, p)) continue;
        double g[2];
        bf_grad_of<NT>(s, v, D, v.scal - s.o_scal + D.oF, p, -1, nullptr, g);
        tot[0] += g[0];
        tot[1] += g[1];
    }
    if (threadIdx.x == 0) {
        v.sg[p * 2] = tot[0];
        v.sg[p * 2 + 1] = tot[1];
    }
    __syncthreads();
}

// ───────────────────────── refresh ──────────────────────────────────────

// Drift refresh of particle p: its determinant derivatives from A and the
// committed rows, and its k-space derivatives from ρ(k) and its phases (left
// in co/so for the ratio).
template <int NT>
__device__ void refresh_particle(const DevSys& s, const Smem& v, const double* grec, int p) {
    const int b = block_of(s, p);
    const bool ks = kspace_of(s, p);
    if (ks) {
        const double th[2] = {s.recip[0] * v.pos[p * 2] + s.recip[1] * v.pos[p * 2 + 1],
                              s.recip[2] * v.pos[p * 2] + s.recip[3] * v.pos[p * 2 + 1]};
        const int m[2] = {s.m1J, s.m2J};
        ladders<NT>(th, m, 2, v.lad);
    }
    double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (b >= 0 && s.cplx) {
        // acc[0..1] Re G, [2..3] Re Lraw, [8..9] Im G, [10..11] Im Lraw
        const DevBlock& B = s.blocks[b];
        const int N = B.n, kr = p - B.first;
        const double* Ar = v.scal - s.o_scal + B.oA;
        const double* Ai = Ar + ((N * N + 3) & ~3);
        for (int m = threadIdx.x; m < N; m += NT) {
            double cs, sn, R[2] = {0, 0};
            c_orb(B, m, v.pos + p * 2, cs, sn);
            c_accumulate(B, m, Ar[m * N + kr], Ai[m * N + kr], cs, sn, R, acc + 0, acc + 8, acc + 2,
                         acc + 10);
        }
    } else if (b >= 0) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, kr = p - B.first;
        const double* A = v.scal - s.o_scal + B.oA;
        const double2* Dg = reinterpret_cast<const double2*>(grec + B.oDg + kr * N * 2);
        const double2* Dl = reinterpret_cast<const double2*>(grec + B.oDl + kr * N * 2);
        for (int m = threadIdx.x; m < N; m += NT) {
            const double a = A[m * N + kr];
            const double2 g = Dg[m];
            const double2 l = Dl[m];
            acc[0] += a * g.x;
            acc[1] += a * g.y;
            acc[2] += a * l.x;
            acc[3] += a * l.y;
        }
    }
    if (ks) {
        __syncthreads();
        const int gp = s.group_of[p];
        for (int k = threadIdx.x; k < s.nkJ; k += NT) {
            double c, sn;
            phase_k(s, v.lad, v.lad + kLad, k, c, sn);
            v.co[k] = c;
            v.so[k] = sn;
            kspace_particle_k(s, v, p, gp, k, c, sn, acc + 4);
        }
    }
    if (s.cplx) block_sum<NT>(acc, v.red);
    else block_sum<NT>(reinterpret_cast<double(&)[8]>(acc), v.red);
    if (threadIdx.x == 0) {
        if (b >= 0 && s.cplx) {
            for (int d = 0; d < 2; ++d) {
                const double gr = acc[d], gi = acc[8 + d];
                v.sg[p * 2 + d] = gr;
                v.pg[p * 2 + d] = gi;
                v.sl[p * 2 + d] = acc[2 + d] - (gr * gr - gi * gi);
                v.pl[p * 2 + d] = acc[10 + d] - 2.0 * gr * gi;
            }
        } else if (b >= 0) {
            v.sg[p * 2 + 0] = acc[0];
            v.sg[p * 2 + 1] = acc[1];
            v.sl[p * 2 + 0] = acc[2] - acc[0] * acc[0];
            v.sl[p * 2 + 1] = acc[3] - acc[1] * acc[1];
        }
        if (ks) {
            v.kg[p * 2 + 0] = acc[4];
            v.kg[p * 2 + 1] = acc[5];
            v.kl[p * 2 + 0] = acc[6];
            v.kl[p * 2 + 1] = acc[7];
        }
    }
    __syncthreads();
    if (s.nbf > 0) bf_refresh_particle<NT>(s, v, p);
}

// ───────────────────────── one-warp helpers ─────────────────────────────
//
// The one-warp sweep (alea_fast.cu) gives lane l the items l, l + 32, ...,
// l + 32(S-1) of each list (partners, orbital rows, k-vectors, particles) and
// keeps per-item intermediates in registers.  Its reductions leave identical
// totals on every lane, so decisions taken from them are warp-uniform.

constexpr unsigned kAllLanes = 0xffffffffu;

// Reduce-scatter of K doubles (K = 4, 8 or 16) across the warp in K shuffles:
// lane l returns the total of value l / (32 / K).  Each level sends half of
// the values still held to the partner lane and keeps the other half.
template <int K>
__device__ __forceinline__ double warp_reduce_scatter(double (&v)[K]) {
    static_assert(K == 4 || K == 8 || K == 16, "K must be 4, 8 or 16");
    const int lane = threadIdx.x & 31;
    int o = 16;
#pragma unroll
    for (int half = K / 2; half >= 1; half /= 2, o /= 2) {
        const bool hi = (lane & o) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            const double send = hi ? v[i] : v[i + half];
            const double keep = hi ? v[i + half] : v[i];
            v[i] = keep + __shfl_xor_sync(kAllLanes, send, o);
        }
    }
    double t = v[0];
    for (; o > 0; o /= 2) t += __shfl_xor_sync(kAllLanes, t, o);
    return t;
}

// All-reduce of K doubles: reduce-scatter, then one broadcast per value.
template <int K>
__device__ __forceinline__ void warp_allsum(double (&v)[K]) {
    const double t = warp_reduce_scatter<K>(v);
#pragma unroll
    for (int i = 0; i < K; ++i) v[i] = __shfl_sync(kAllLanes, t, i * (32 / K));
}

__device__ __forceinline__ double warp_max(double x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(kAllLanes, x, o));
    return x;
}

// Phase e^{ik·r} of the k-vectors of a list visited in order: a k that
// follows its predecessor by one step of n2 multiplies the previous phase by
// e^{iθ2} (θ2 = b2·r); any other k starts afresh from sincos(n1 θ1 + n2 θ2).
struct PhaseWalk {
    int n1 = -(1 << 30), n2 = 0;
    __device__ __forceinline__ void next(int m1, int m2, double th1, double th2, double e2r, double e2i,
                                         double& c, double& sn) {
        if (m1 == n1 && m2 == n2 + 1) {
            const double cr = c * e2r - sn * e2i;
            sn = fma(c, e2i, sn * e2r);
            c = cr;
        } else {
            sincos(fma(static_cast<double>(m2), th2, static_cast<double>(m1) * th1), &sn, &c);
        }
        n1 = m1;
        n2 = m2;
    }
};

// k-space gradient and Laplacian of every particle (one warp): the image
// terms' weights and the partner densities are folded per group into
// E_g(k) = Σ_t w_t(k) ρ_{g'(t)}(k) in `work`; the self weight
// S_g(k) = Σ_{t same-group} w_t(k) is summed per lane from the weights.  Lane
// slot i then walks the k list once with its own phase.
template <int S>
__device__ void kspace_refresh_warp(const DevSys& s, const Smem& v) {
    const int np = s.np, nk = s.nkJ, ng = s.ngroups;
    double* E = v.work;   // [g][2][nk]: Re E, Im E
    for (int e = threadIdx.x; e < ng * nk; e += 32) {
        const int g = e / nk, q = e - g * nk;
        double er = 0.0, ei = 0.0;
        for (int t = 0; t < s.nterms; ++t) {
            const DevTerm& T = s.terms[t];
            if (!T.image || !in_term(T, s.gfirst[g])) continue;
            const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
            const int go = T.same0 ? g : (g == ga ? gb : ga);
            const double w = T.kw[q];
            er += w * v.rho[go * 2 * nk + q];
            ei += w * v.rho[go * 2 * nk + nk + q];
        }
        E[(g * 2 + 0) * nk + q] = er;
        E[(g * 2 + 1) * nk + q] = ei;
    }
    __syncwarp();
    double th1[S], th2[S], e2r[S], e2i[S], c[S], sn[S], acc[S][4];
    int gi[S];
    unsigned selfmask[S];   // same-group image terms of the slot's group: S_g(k) = Σ their w(k)
    bool on[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int i = threadIdx.x + 32 * j;
        on[j] = i < np && kspace_of(s, i);
        gi[j] = i < np ? s.group_of[i] : 0;
        selfmask[j] = 0u;
        for (int t = 0; t < s.nterms; ++t)
            if (s.terms[t].image && s.terms[t].same0 && in_term(s.terms[t], s.gfirst[gi[j]]))
                selfmask[j] |= 1u << t;
        const double x = i < np ? v.pos[i * 2] : 0.0, y = i < np ? v.pos[i * 2 + 1] : 0.0;
        th1[j] = s.recip[0] * x + s.recip[1] * y;
        th2[j] = s.recip[2] * x + s.recip[3] * y;
        sincos(th2[j], &e2i[j], &e2r[j]);
        c[j] = 1.0;
        sn[j] = 0.0;
        acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
    }
    PhaseWalk walk[S];
    for (int q = 0; q < nk; ++q) {
        const int m1 = s.n1J[q], m2 = s.n2J[q];
        const double kx = s.kxJ[q], ky = s.kyJ[q], kx2 = s.kx2J[q], ky2 = s.ky2J[q];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            walk[j].next(m1, m2, th1[j], th2[j], e2r[j], e2i[j], c[j], sn[j]);
            const double* Eg = E + gi[j] * 2 * nk;
            const double er = Eg[q], ei = Eg[nk + q];
            double sw = 0.0;
            for (unsigned bits = selfmask[j]; bits; bits &= bits - 1) sw += s.terms[__ffs(bits) - 1].kw[q];
            const double g = 2.0 * (c[j] * ei - sn[j] * er);
            const double l = 2.0 * (sw - (c[j] * er + sn[j] * ei));
            acc[j][0] += kx * g;
            acc[j][1] += ky * g;
            acc[j][2] += kx2 * l;
            acc[j][3] += ky2 * l;
        }
    }
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int i = threadIdx.x + 32 * j;
        if (!on[j]) continue;
        v.kg[i * 2] = acc[j][0];
        v.kg[i * 2 + 1] = acc[j][1];
        v.kl[i * 2] = acc[j][2];
        v.kl[i * 2 + 1] = acc[j][3];
    }
    __syncwarp();
}

// Ewald reciprocal sum Σ_k w_k |ρ(k)|², ρ(k) = Σ_i q_i e^{ik·r_i}, on one
// warp: lane slot i walks the k list with its particle's phase; eight k at a
// time, the lanes' (Re, Im) contributions meet in a 16-value reduce-scatter
// and land in `work`.  Returns this lane's share of the sum.
template <int S>
__device__ double ewald_recip_warp(const DevSys& s, const Smem& v) {
    const int np = s.np, nk = s.enk;
    const int lane = threadIdx.x & 31;
    double* rk = v.work;   // [k][2]
    double qc[S], th1[S], th2[S], e2r[S], e2i[S], c[S], sn[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int i = lane + 32 * j;
        qc[j] = i < np ? s.charge[i] : 0.0;
        const double x = i < np ? v.pos[i * 2] : 0.0, y = i < np ? v.pos[i * 2 + 1] : 0.0;
        th1[j] = s.recip[0] * x + s.recip[1] * y;
        th2[j] = s.recip[2] * x + s.recip[3] * y;
        sincos(th2[j], &e2i[j], &e2r[j]);
        c[j] = 1.0;
        sn[j] = 0.0;
    }
    PhaseWalk walk[S];
    for (int kb = 0; kb < nk; kb += 8) {
        double val[16];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            const int q = kb + t;
            double vr = 0.0, vi = 0.0;
            if (q < nk) {
                const int m1 = s.en1[q], m2 = s.en2[q];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    walk[j].next(m1, m2, th1[j], th2[j], e2r[j], e2i[j], c[j], sn[j]);
                    vr = fma(qc[j], c[j], vr);
                    vi = fma(qc[j], sn[j], vi);
                }
            }
            val[2 * t] = vr;
            val[2 * t + 1] = vi;
        }
        const double tot = warp_reduce_scatter<16>(val);
        const int idx = lane >> 1;
        if ((lane & 1) == 0 && kb + (idx >> 1) < nk) rk[(kb + (idx >> 1)) * 2 + (idx & 1)] = tot;
    }
    __syncwarp();
    double e = 0.0;
    for (int q = lane; q < nk; q += 32) e += s.ew[q] * (rk[q * 2] * rk[q * 2] + rk[q * 2 + 1] * rk[q * 2 + 1]);
    __syncwarp();
    return e;
}

// Ewald real-space sum Σ_{i<j} q_i q_j [1/(ε r) - V_long(r)] (r < r_cut) on
// one warp: three pairs per lane in flight, no branch in the pair body.
__device__ __forceinline__ double ewald_real_warp(const DevSys& s, const Smem& v, const int2* pairs,
                                                  int npair) {
    double e0 = 0.0, e1 = 0.0, e2 = 0.0;
    const int lane = threadIdx.x & 31;
    for (int q0 = lane; q0 < npair; q0 += 96) {
        double acc3[3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const int q = q0 + 32 * u;
            const bool on = q < npair;
            const int2 pq = on ? pairs[q] : make_int2(0, 0);
            const double coeff = on ? ldg_keep(s.charge + pq.x) * ldg_keep(s.charge + pq.y) : 0.0;
            double dx, dy;
            const double r = on ? fold2(s, v.pos[pq.x * 2], v.pos[pq.x * 2 + 1], v.pos[pq.y * 2],
                                        v.pos[pq.y * 2 + 1], dx, dy)
                                : 1.0;
            const double t = coeff * (s.e_inv_eps / r - spline1(s.esp, r));
            acc3[u] = (on && coeff != 0.0 && r < s.e_rcut) ? t : 0.0;
        }
        e0 += acc3[0];
        e1 += acc3[1];
        e2 += acc3[2];
    }
    return e0 + e1 + e2;
}

// Every particle's determinant and k-space derivatives (refresh_derivatives).
// S > 0: the one-warp form (real determinants, lane-owned rows).
template <int NT, int S = 0>
__device__ void refresh_all(const DevSys& s, const Smem& v, const double* grec) {
    const int np = s.np;
    if constexpr (S > 0) {
        if (s.cplx) c_refresh_all<32>(s, v);   // complex rows from the positions, one particle per lane
        for (int b = 0; b < (s.cplx ? 0 : s.nblocks); ++b) {
            const DevBlock& B = s.blocks[b];
            const int N = B.n;
            const double* A = v.scal - s.o_scal + B.oA;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                const int kr = static_cast<int>(threadIdx.x) + 32 * j;
                if (kr >= N) continue;
                const double2* rg = reinterpret_cast<const double2*>(grec + B.oDg) + kr * N;
                const double2* rl = reinterpret_cast<const double2*>(grec + B.oDl) + kr * N;
                double g0 = 0.0, g1 = 0.0, l0 = 0.0, l1 = 0.0;
#pragma unroll 4
                for (int m = 0; m < N; ++m) {
                    const double a = A[m * N + kr];
                    const double2 dg = rg[m], dl = rl[m];
                    g0 += a * dg.x;
                    g1 += a * dg.y;
                    l0 += a * dl.x;
                    l1 += a * dl.y;
                }
                const int part = B.first + kr;
                v.sg[part * 2] = g0;
                v.sg[part * 2 + 1] = g1;
                v.sl[part * 2] = l0 - g0 * g0;
                v.sl[part * 2 + 1] = l1 - g1 * g1;
            }
        }
        if (s.nkJ > 0) kspace_refresh_warp<S>(s, v);
        __syncwarp();
        return;
    }
    if (s.nbf > 0) bf_refresh_all<NT>(s, v, false);
    if (s.cplx) c_refresh_all<NT>(s, v);
    for (int b = 0; b < (s.cplx ? 0 : s.nblocks); ++b) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n;
        const double* A = v.scal - s.o_scal + B.oA;
        const double* Dg = grec + B.oDg;
        const double* Dl = grec + B.oDl;
        for (int t = threadIdx.x; t < N * 2; t += NT) {
            const int kr = t >> 1, d = t & 1;
            double g = 0.0, l = 0.0;
            for (int m = 0; m < N; ++m) {
                const double a = A[m * N + kr];
                g += a * Dg[(kr * N + m) * 2 + d];
                l += a * Dl[(kr * N + m) * 2 + d];
            }
            const int part = B.first + kr;
            v.sg[part * 2 + d] = g;
            v.sl[part * 2 + d] = l - g * g;
        }
    }
    if (s.nkJ > 0) {
        const int m[2] = {s.m1J, s.m2J};
        for (int i = 0; i < np; ++i) {
            if (!kspace_of(s, i)) continue;
            __syncthreads();
            const double th[2] = {s.recip[0] * v.pos[i * 2] + s.recip[1] * v.pos[i * 2 + 1],
                                  s.recip[2] * v.pos[i * 2] + s.recip[3] * v.pos[i * 2 + 1]};
            ladders<NT>(th, m, 2, v.lad);
            __syncthreads();
            const int gi = s.group_of[i];
            double acc[4] = {0, 0, 0, 0};
            for (int k = threadIdx.x; k < s.nkJ; k += NT) {
                double c, sn;
                phase_k(s, v.lad, v.lad + kLad, k, c, sn);
                kspace_particle_k(s, v, i, gi, k, c, sn, acc);
            }
            block_sum<NT>(acc, v.red);
            if (threadIdx.x == 0) {
                v.kg[i * 2] = acc[0];
                v.kg[i * 2 + 1] = acc[1];
                v.kl[i * 2] = acc[2];
                v.kl[i * 2 + 1] = acc[3];
            }
        }
    }
    __syncthreads();
}

// ───────────────────────── ratio ────────────────────────────────────────

// ln|ψ'/ψ| of moving p to v.newpos.  `have_old` says whether co/so already
// hold p's current phases (a drift refresh computed them).  Leaves in misc:
// R, scale, the log ratio, the phase and the determinant, pair and k-space
// parts of ∇ln ψ and ∂² ln ψ of p at the proposal; in shared memory: the new
// orbital row, the per-partner radial derivatives (rad) and geometry (geo),
// and p's new phases (cn/sn).
template <int NT>
__device__ void ratio_step(const DevSys& s, const Smem& v, int p, bool have_old) {
    const int np = s.np;
    const int b = block_of(s, p);
    const bool ks = kspace_of(s, p);
    // acc: 0 R (Re R), 1 Σ|terms| (Im R when complex), 2-5 determinant ∇, ∂² of p
    // (Re parts), 6 Jastrow log ratio, 7-10 pair ∇, ∂², 11-14 k-space ∇, ∂²,
    // 15-18 determinant Im ∇, Im ∂² (complex)
    double acc[19];
#pragma unroll
    for (int i = 0; i < 19; ++i) acc[i] = 0.0;
    // backflow determinants first: their proposal uses the work area that the
    // pair loop below fills with partner scratch
    for (int d = 0; d < s.nbf; ++d)
        if (bf_affects(s.bf[d], p)) bf_propose<NT>(s, v, d, p);
    if (ks) {
        const double* r = v.pos + p * 2;
        const double th[4] = {s.recip[0] * v.newpos[0] + s.recip[1] * v.newpos[1],
                              s.recip[2] * v.newpos[0] + s.recip[3] * v.newpos[1],
                              s.recip[0] * r[0] + s.recip[1] * r[1],
                              s.recip[2] * r[0] + s.recip[3] * r[1]};
        const int m[4] = {s.m1J, s.m2J, s.m1J, s.m2J};
        ladders<NT>(th, m, have_old ? 2 : 4, v.lad);
    }
    if (b >= 0 && s.cplx) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, jrow = p - B.first;
        const double* Ar = v.scal - s.o_scal + B.oA;
        const double* Ai = Ar + ((N * N + 3) & ~3);
        for (int m = threadIdx.x; m < N; m += NT) {
            double cs, sn;
            c_orb(B, m, v.newpos, cs, sn);
            v.nval[m] = cs;
            v.nval[N + m] = sn;
            c_accumulate(B, m, Ar[m * N + jrow], Ai[m * N + jrow], cs, sn, acc, acc + 2, acc + 15,
                         acc + 4, acc + 17);
        }
    } else if (b >= 0) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, jrow = p - B.first;
        const double* A = v.scal - s.o_scal + B.oA;
        for (int m = threadIdx.x; m < N; m += NT) {
            double val, g[3], l[3];
            orbital(s, B, m, v.newpos, val, g, l);
            v.nval[m] = val;
            v.ngrad[m * 2 + 0] = g[0];
            v.ngrad[m * 2 + 1] = g[1];
            v.nlap[m * 2 + 0] = l[0];
            v.nlap[m * 2 + 1] = l[1];
            const double a = A[m * N + jrow];
            const double term = a * val;
            acc[0] += term;
            acc[1] += fabs(term);
            acc[2] += a * g[0];
            acc[3] += a * g[1];
            acc[4] += a * l[0];
            acc[5] += a * l[1];
        }
    }
    for (int k = threadIdx.x; k < np; k += NT) {
        if (k == p) continue;
        const unsigned cm = coupling(s, p, k);
        if (!cm) continue;
        double dn[3], dold[3];
        const double rn = fold_dist(s, v.newpos, v.pos + k * 2, dn);
        const double ro = fold_dist(s, v.pos + p * 2, v.pos + k * 2, dold);
        double* geo = v.geo + k * 6;
        geo[0] = dn[0];
        geo[1] = dn[1];
        geo[2] = rn;
        geo[3] = dold[0];
        geo[4] = dold[1];
        geo[5] = ro;
        double du_o = 0.0, d2u_o = 0.0, du_n = 0.0, d2u_n = 0.0;
        for (unsigned bits = cm; bits; bits &= bits - 1) {
            const DevTerm& T = s.terms[__ffs(bits) - 1];
            double uo, duo, d2uo, un, dun, d2un;
            radial(T, ro, uo, duo, d2uo);
            radial(T, rn, un, dun, d2un);
            acc[6] += un - uo;
            du_o += duo;
            d2u_o += d2uo;
            du_n += dun;
            d2u_n += d2un;
        }
        double* rad = v.rad + k * 4;
        rad[0] = du_o;
        rad[1] = d2u_o;
        rad[2] = du_n;
        rad[3] = d2u_n;
        const double invr = 1.0 / rn;
        for (int d = 0; d < 2; ++d) {
            const double dor = dn[d] * invr;
            acc[7 + d] += du_n * dor;
            acc[9 + d] += d2u_n * dor * dor + du_n * invr * (1.0 - dor * dor);
        }
    }
    if (ks) {
        __syncthreads();
        const int nk = s.nkJ;
        const int gp = s.group_of[p];
        for (int k = threadIdx.x; k < nk; k += NT) {
            double c, sn, co, so;
            phase_k(s, v.lad, v.lad + kLad, k, c, sn);
            if (have_old) {
                co = v.co[k];
                so = v.so[k];
            } else {
                phase_k(s, v.lad + 2 * kLad, v.lad + 3 * kLad, k, co, so);
                v.co[k] = co;
                v.so[k] = so;
            }
            v.cn[k] = c;
            v.sn[k] = sn;
            for (int t = 0; t < s.nterms; ++t) {
                const DevTerm& T = s.terms[t];
                if (!T.image || !in_term(T, p)) continue;
                const double w = T.kw[k];
                const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
                const double* mr = v.rho + gp * 2 * nk;
                if (T.same0) {
                    const double qr = mr[k] + c - co;
                    const double qi = mr[nk + k] + sn - so;
                    acc[6] += w * (qr * qr + qi * qi - mr[k] * mr[k] - mr[nk + k] * mr[nk + k]);
                    kterm(s, w, k, c, sn, qr, qi, 1.0, acc + 11);
                } else {
                    const int go = gp == ga ? gb : ga;
                    const double* orr = v.rho + go * 2 * nk;
                    acc[6] += 2.0 * w * ((c - co) * orr[k] + (sn - so) * orr[nk + k]);
                    kterm(s, w, k, c, sn, orr[k], orr[nk + k], 0.0, acc + 11);
                }
            }
        }
    }
    if (s.cplx) block_sum<NT>(acc, v.red);
    else block_sum<NT>(reinterpret_cast<double(&)[15]>(acc), v.red);
    if (threadIdx.x == 0) {
        double logr = acc[6], phase = 0.0, sgx = 0.0, sgy = 0.0, slx = 0.0, sly = 0.0;
        double pgx = 0.0, pgy = 0.0, plx = 0.0, ply = 0.0, logdr = 0.0;
        if (b >= 0 && s.cplx) {
            // R = Σ A[m][j] φ_m(r'); ∇ln ψ' = G/R, ∂²ln ψ' = Lraw/R - (G/R)²
            const double rr = acc[0], ri = acc[1];
            const double a2 = rr * rr + ri * ri;
            logdr = log(fmax(sqrt(a2), 1e-300));
            phase = atan2(ri, rr);
            const double ir = a2 > 0.0 ? rr / a2 : 0.0, ii = a2 > 0.0 ? -ri / a2 : 0.0;
            double gr[2], gi[2], lr[2], li[2];
            for (int d = 0; d < 2; ++d) {
                gr[d] = acc[2 + d] * ir - acc[15 + d] * ii;
                gi[d] = acc[2 + d] * ii + acc[15 + d] * ir;
                lr[d] = acc[4 + d] * ir - acc[17 + d] * ii - (gr[d] * gr[d] - gi[d] * gi[d]);
                li[d] = acc[4 + d] * ii + acc[17 + d] * ir - 2.0 * gr[d] * gi[d];
            }
            sgx = gr[0]; sgy = gr[1]; slx = lr[0]; sly = lr[1];
            pgx = gi[0]; pgy = gi[1]; plx = li[0]; ply = li[1];
        } else if (b >= 0) {
            const double R = acc[0];
            logdr = log(fmax(fabs(R), 1e-300));
            if (R < 0.0) phase = kPi;
            const double invR = (R != 0.0) ? 1.0 / R : 0.0;
            sgx = invR * acc[2];
            sgy = invR * acc[3];
            slx = invR * acc[4] - sgx * sgx;
            sly = invR * acc[5] - sgy * sgy;
        }
        for (int d = 0; d < s.nbf; ++d) {   // BackflowSlaterDeterminant::ratio_batch
            const DevBF& D = s.bf[d];
            if (!bf_affects(D, p)) continue;
            const double* pm = v.scal - s.o_scal + D.pM;
            const double* ls = v.scal - s.o_scal + D.oLS;
            if (pm[2] == 0.0) {
                logdr += -700.0;   // a singular proposal is never accepted
                continue;
            }
            logdr += pm[0] - ls[0];
            if (pm[1] * ls[1] < 0.0) phase += kPi;
            sgx += pm[3];
            sgy += pm[4];
        }
        logr += logdr;
        v.misc[M_LOGDR] = logdr;
        v.misc[M_RI] = s.cplx ? acc[1] : 0.0;
        v.misc[M_PGX] = pgx;
        v.misc[M_PGY] = pgy;
        v.misc[M_PLX] = plx;
        v.misc[M_PLY] = ply;
        v.misc[M_R] = acc[0];
        v.misc[M_SCALE] = acc[1];
        v.misc[M_LOGR] = logr;
        v.misc[M_PHASE] = phase;
        v.misc[M_SGX] = sgx;
        v.misc[M_SGY] = sgy;
        v.misc[M_SLX] = slx;
        v.misc[M_SLY] = sly;
        v.misc[M_JGX] = acc[7];
        v.misc[M_JGY] = acc[8];
        v.misc[M_JLX] = acc[9];
        v.misc[M_JLY] = acc[10];
        v.misc[M_KGX] = acc[11];
        v.misc[M_KGY] = acc[12];
        v.misc[M_KLX] = acc[13];
        v.misc[M_KLY] = acc[14];
    }
    __syncthreads();
}

// ───────────────────────── commit ───────────────────────────────────────

template <int NT>
__device__ void commit_step(const DevSys& s, const Smem& v, double* grec, int p) {
    const int np = s.np;
    const int b = block_of(s, p);
    // pair terms first (their scratch shares space with the rebuild's work
    // matrix): partner gradients and Laplacians, eager as in the reference
    for (int k = threadIdx.x; k < np; k += NT) {
        if (k == p || !coupling(s, p, k)) continue;
        const double* geo = v.geo + k * 6;
        const double* rad = v.rad + k * 4;
        const double irn = 1.0 / geo[2], iro = 1.0 / geo[5];
        for (int d = 0; d < 2; ++d) {
            const double dor_old = -geo[3 + d] * iro, dor_new = -geo[d] * irn;
            const double g_old = rad[0] * dor_old, g_new = rad[2] * dor_new;
            v.jg[k * 2 + d] += g_new - g_old;
            const double lap_old = rad[1] * dor_old * dor_old + rad[0] * iro * (1.0 - dor_old * dor_old);
            const double lap_new = rad[3] * dor_new * dor_new + rad[2] * irn * (1.0 - dor_new * dor_new);
            v.jl[k * 2 + d] += lap_new - lap_old;
        }
    }
    // k-space: ρ of p's group follows the move; partners refresh on their next read
    if (kspace_of(s, p)) {
        const int nk = s.nkJ;
        double* mr = v.rho + s.group_of[p] * 2 * nk;
        for (int k = threadIdx.x; k < nk; k += NT) {
            mr[k] += v.cn[k] - v.co[k];
            mr[nk + k] += v.sn[k] - v.so[k];
        }
    }
    // complex determinant: complex Sherman-Morrison, rebuilt by Gauss-Jordan
    // from recomputed rows every 64 updates or at a small or nonfinite ratio
    if (b >= 0 && s.cplx) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, jrow = p - B.first;
        double* Ar = v.scal - s.o_scal + B.oA;
        double* Ai = Ar + ((N * N + 3) & ~3);
        double* bs = v.scal + S_BLOCK0 + 3 * b;
        const double rr = v.misc[M_R], ri = v.misc[M_RI];
        const double a2 = rr * rr + ri * ri;
        const double ir = rr / a2, ii = -ri / a2;
        const double* nr = v.nval;
        const double* ni = v.nval + N;
        for (int c = threadIdx.x; c < N; c += NT) {
            double pr = 0.0, pi = 0.0;
            for (int m = 0; m < N; ++m) {
                const double xr = nr[m], xi = ni[m], ar = Ar[m * N + c], ai = Ai[m * N + c];
                pr += xr * ar - xi * ai;
                pi += xr * ai + xi * ar;
            }
            v.rowp[c] = pr - (c == jrow ? 1.0 : 0.0);
            v.rowp[N + c] = pi;
            const double cr = Ar[c * N + jrow], ci = Ai[c * N + jrow];
            v.col[c] = cr * ir - ci * ii;   // A[c][j] / R
            v.col[N + c] = cr * ii + ci * ir;
        }
        if (threadIdx.x == 0) {
            bs[1] += 1.0;
            const bool rebuild = bs[1] >= 64.0 || !isfinite(a2) || sqrt(a2) < 1e-5;
            v.misc[M_REBUILD] = rebuild ? 1.0 : 0.0;
        }
        __syncthreads();
        const double old_log = bs[0];
        const bool rebuild = v.misc[M_REBUILD] != 0.0;
        if (rebuild) {
            c_gj_rebuild<NT>(s, v, b, p, v.newpos);
        } else {
            for_each_elem<NT>(N, [&](int a, int c) {
                const double fr = v.col[a], fi = v.col[N + a];
                const double qr = v.rowp[c], qi = v.rowp[N + c];
                Ar[a * N + c] -= fr * qr - fi * qi;
                Ai[a * N + c] -= fr * qi + fi * qr;
            });
            __syncthreads();
        }
        // the moved particle's derivatives at the committed inverse
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int m = threadIdx.x; m < N; m += NT) {
            double R[2] = {0, 0};
            c_accumulate(B, m, Ar[m * N + jrow], Ai[m * N + jrow], nr[m], ni[m], R, acc + 0, acc + 4,
                         acc + 2, acc + 6);
        }
        block_sum<NT>(acc, v.red);
        if (threadIdx.x == 0) {
            if (rebuild) {
                bs[0] = v.misc[M_LOGDET];
                bs[1] = 0.0;
                if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
            } else {
                bs[0] = old_log + v.misc[M_LOGDR];
            }
            v.scal[S_LOGPSI] += bs[0] - old_log;
            for (int d = 0; d < 2; ++d) {
                const double gr = acc[d], gi = acc[4 + d];
                v.sg[p * 2 + d] = gr;
                v.pg[p * 2 + d] = gi;
                v.sl[p * 2 + d] = acc[2 + d] - (gr * gr - gi * gi);
                v.pl[p * 2 + d] = acc[6 + d] - 2.0 * gr * gi;
            }
        }
    } else if (b >= 0) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, jrow = p - B.first;
        double* A = v.scal - s.o_scal + B.oA;
        double* bs = v.scal + S_BLOCK0 + 3 * b;
        double* D = grec + B.oD;
        double* Dg = grec + B.oDg;
        double* Dl = grec + B.oDl;
        double* rabs = v.scal - s.o_scal + B.orabs;
        const double R = v.misc[M_R];
        for (int c = threadIdx.x; c < N; c += NT) {
            double prod = 0.0;
            for (int m = 0; m < N; ++m) prod += v.nval[m] * A[m * N + c];
            v.rowp[c] = prod - (c == jrow ? 1.0 : 0.0);
            v.col[c] = A[c * N + jrow] / R;   // factor of row c of the update
            D[jrow * N + c] = v.nval[c];
            reinterpret_cast<double2*>(Dg + jrow * N * 2)[c] =
                make_double2(v.ngrad[c * 2 + 0], v.ngrad[c * 2 + 1]);
            reinterpret_cast<double2*>(Dl + jrow * N * 2)[c] =
                make_double2(v.nlap[c * 2 + 0], v.nlap[c * 2 + 1]);
        }
        if (threadIdx.x == 0) {
            bs[1] += 1.0;
            const bool rebuild = bs[1] >= 64.0 || !isfinite(R) || fabs(R) < 1e-5 || bs[2] > 1e8 ||
                                 fabs(R) <= 1e4 * kEps * v.misc[M_SCALE];
            v.misc[M_REBUILD] = rebuild ? 1.0 : 0.0;
            double rd = 0.0;
            for (int m = 0; m < N; ++m) rd += fabs(v.nval[m]);
            rabs[jrow] = rd;
        }
        __syncthreads();
        const double old_log = bs[0];
        bool rebuild = v.misc[M_REBUILD] != 0.0;
        if (rebuild) {
            gj_rebuild<NT>(s, v, grec, b);
        } else {
            for_each_elem<NT>(N, [&](int a, int c) { A[a * N + c] = A[a * N + c] - v.col[a] * v.rowp[c]; });
            __syncthreads();
        }
        double ra = 0.0, rdm = 0.0;
        for (int a = threadIdx.x; a < N; a += NT) {
            double t = 0.0;
            for (int c = 0; c < N; ++c) t += fabs(A[a * N + c]);
            ra = fmax(ra, t);
            rdm = fmax(rdm, rabs[a]);
        }
        const double norm_a = block_max<NT>(ra, v.red);
        const double norm_d = block_max<NT>(rdm, v.red);
        const double cond = norm_d * norm_a;
        if (!rebuild && (!isfinite(cond) || cond > 1e8)) {
            gj_rebuild<NT>(s, v, grec, b);
            rebuild = true;
        }
        // the moved particle's determinant derivatives at the committed inverse
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int m = threadIdx.x; m < N; m += NT) {
            const double a = A[m * N + jrow];
            acc[0] += a * v.ngrad[m * 2 + 0];
            acc[1] += a * v.ngrad[m * 2 + 1];
            acc[2] += a * v.nlap[m * 2 + 0];
            acc[3] += a * v.nlap[m * 2 + 1];
        }
        block_sum<NT>(acc, v.red);
        if (threadIdx.x == 0) {
            bs[2] = cond;
            if (rebuild) {
                bs[0] = v.misc[M_LOGDET];
                bs[1] = 0.0;
                if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
            } else {
                bs[0] = old_log + log(fabs(R));
            }
            v.scal[S_LOGPSI] += bs[0] - old_log;
            v.sg[p * 2 + 0] = acc[0];
            v.sg[p * 2 + 1] = acc[1];
            v.sl[p * 2 + 0] = acc[2] - acc[0] * acc[0];
            v.sl[p * 2 + 1] = acc[3] - acc[1] * acc[1];
        }
    }
    // backflow determinants: the pending proposal becomes committed
    if (s.nbf > 0) {
        double* sm = v.scal - s.o_scal;
        for (int d = 0; d < s.nbf; ++d) {
            const DevBF& D = s.bf[d];
            if (!bf_affects(D, p)) continue;
            const int N = D.n;
            for (int i = threadIdx.x; i < 2 * N; i += NT) {
                sm[D.oX + i] = sm[D.pX + i];
                sm[D.oF + i] = sm[D.pF + i];
            }
            for (int i = threadIdx.x; i < N * N; i += NT) sm[D.oA + i] = sm[D.pA + i];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double g0 = 0.0, g1 = 0.0;
            for (int d = 0; d < s.nbf; ++d) {
                const DevBF& D = s.bf[d];
                if (!bf_affects(D, p)) continue;
                const double* pm = sm + D.pM;
                double* ls = sm + D.oLS;
                if (pm[2] == 0.0) v.scal[S_ERR] = 1.0;
                v.scal[S_LOGPSI] += pm[0] - ls[0];
                ls[0] = pm[0];
                ls[1] = pm[1];
                g0 += pm[3];
                g1 += pm[4];
            }
            v.sg[p * 2] = g0;          // exact at the committed state
            v.sg[p * 2 + 1] = g1;
            v.sl[p * 2] = 0.0;         // proposal Laplacian skipped (refreshed before E_L)
            v.sl[p * 2 + 1] = 0.0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        v.jg[p * 2 + 0] = v.misc[M_JGX];
        v.jg[p * 2 + 1] = v.misc[M_JGY];
        v.jl[p * 2 + 0] = v.misc[M_JLX];
        v.jl[p * 2 + 1] = v.misc[M_JLY];
        v.kg[p * 2 + 0] = v.misc[M_KGX];
        v.kg[p * 2 + 1] = v.misc[M_KGY];
        v.kl[p * 2 + 0] = v.misc[M_KLX];
        v.kl[p * 2 + 1] = v.misc[M_KLY];
        double r[3] = {v.newpos[0], v.newpos[1], 0.0};
        wrap_pos(s, r);
        v.pos[p * 2 + 0] = r[0];
        v.pos[p * 2 + 1] = r[1];
        v.scal[S_LOGPSI] += v.misc[M_LOGR] - v.misc[M_LOGDR];
    }
    __syncthreads();
    // Wrapping p into the cell moved it by a lattice vector Δ; a twisted
    // plane wave picks up the same phase e^{iθ·Δ} = e^{iq·Δ} for every
    // orbital, so the inverse's column of p is re-gauged by e^{-iq·Δ} to stay
    // the inverse of the rows at the stored positions.
    if (s.cplx && b >= 0) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n, jrow = p - B.first;
        const double dx = v.pos[p * 2] - v.newpos[0], dy = v.pos[p * 2 + 1] - v.newpos[1];
        if (dx != 0.0 || dy != 0.0) {
            double* Ar = v.scal - s.o_scal + B.oA;
            double* Ai = Ar + ((N * N + 3) & ~3);
            double sa, ca;
            sincos(fma(B.k[1], dy, B.k[0] * dx), &sa, &ca);
            for (int m = threadIdx.x; m < N; m += NT) {
                const double ar = Ar[m * N + jrow], ai = Ai[m * N + jrow];
                Ar[m * N + jrow] = ar * ca + ai * sa;
                Ai[m * N + jrow] = ai * ca - ar * sa;
            }
        }
        __syncthreads();
    }
}

// ───────────────────────── local energy ─────────────────────────────────

// E_L from refreshed derivatives: kinetic + Ewald (real, reciprocal,
// constants) + open Coulomb.  Reciprocal ρ(k) accumulates particle by
// particle in `work` (one slot per k, owned by one thread); S > 0 takes the
// one-warp reciprocal sum instead.
template <int NT, int S = 0>
__device__ double local_energy(const DevSys& s, const Smem& v, const int2* pairs, int npair) {
    const int np = s.np;
    double acc[2] = {0.0, 0.0};   // Re, Im E_L
    for (int t = threadIdx.x; t < np * 2; t += NT) {
        const double g = v.sg[t] + v.jg[t] + v.kg[t], l = v.sl[t] + v.jl[t] + v.kl[t];
        acc[0] += -0.5 * s.inv_mass[t] * (l + g * g);
        if (s.cplx) {   // Kinetic::add_phase_terms
            acc[0] += 0.5 * s.inv_mass[t] * v.pg[t] * v.pg[t];
            acc[1] += -0.5 * s.inv_mass[t] * (v.pl[t] + 2.0 * g * v.pg[t]);
        }
    }
    if (s.ewald) {
        if constexpr (S > 0) acc[0] += ewald_real_warp(s, v, pairs, npair);
        for (int q = threadIdx.x; q < (S > 0 ? 0 : npair); q += NT) {
            const int2 pq = pairs[q];
            const double coeff = s.charge[pq.x] * s.charge[pq.y];
            if (coeff == 0.0) continue;
            double del[3];
            const double r = fold_dist(s, v.pos + pq.x * 2, v.pos + pq.y * 2, del);
            if (r < s.e_rcut) acc[0] += coeff * (s.e_inv_eps / r - spline1(s.esp, r));
        }
        if constexpr (S > 0) {
            acc[0] += ewald_recip_warp<S>(s, v);
        } else {
        double* rr = v.work;
        double* ri = v.work + s.enk;
        for (int k = threadIdx.x; k < s.enk; k += NT) rr[k] = ri[k] = 0.0;
        const int m[2] = {s.e_m1, s.e_m2};
        for (int i = 0; i < np; ++i) {
            const double q = s.charge[i];
            if (q == 0.0) continue;
            __syncthreads();
            const double th[2] = {s.recip[0] * v.pos[i * 2] + s.recip[1] * v.pos[i * 2 + 1],
                                  s.recip[2] * v.pos[i * 2] + s.recip[3] * v.pos[i * 2 + 1]};
            ladders<NT>(th, m, 2, v.lad);
            __syncthreads();
            for (int k = threadIdx.x; k < s.enk; k += NT) {
                double ar, ai, br, bi;
                ladder_pick(v.lad, s.en1[k], ar, ai);
                ladder_pick(v.lad + kLad, s.en2[k], br, bi);
                rr[k] += q * (ar * br - ai * bi);
                ri[k] += q * (ar * bi + ai * br);
            }
        }
        for (int k = threadIdx.x; k < s.enk; k += NT) acc[0] += s.ew[k] * (rr[k] * rr[k] + ri[k] * ri[k]);
        }
    }
    for (int c = 0; c < s.ncoul; ++c) {
        const int af = s.coul[c][0], al = s.coul[c][1], bf = s.coul[c][2], bl = s.coul[c][3];
        const bool same = af == bf && al == bl;
        const int na = al - af, nb = bl - bf;
        const int tot = same ? na * na : na * nb;
        for (int q = threadIdx.x; q < tot; q += NT) {
            const int i = af + q / (same ? na : nb), j = (same ? af : bf) + q % (same ? na : nb);
            if (same && j <= i) continue;
            double del[3];
            const double r = fold_dist(s, v.pos + i * 2, v.pos + j * 2, del);
            acc[0] += s.coul_coef[c] / r;
        }
    }
    // C r^-p at the minimum image (the continuum tail is a constant below)
    for (int c = 0; c < s.nip; ++c) {
        const int af = s.ip[c][0], al = s.ip[c][1], bf = s.ip[c][2], bl = s.ip[c][3];
        const bool same = af == bf && al == bl;
        const int na = al - af, nb = bl - bf;
        const int tot = same ? na * na : na * nb;
        for (int q = threadIdx.x; q < tot; q += NT) {
            const int i = af + q / (same ? na : nb), j = (same ? af : bf) + q % (same ? na : nb);
            if (same && j <= i) continue;
            double del[3];
            const double r = fold_dist(s, v.pos + i * 2, v.pos + j * 2, del);
            if (s.ip_pint[c] > 0) {
                const double inv_r = 1.0 / r;
                double inv_rp = inv_r;
                for (int k = 1; k < s.ip_pint[c]; ++k) inv_rp *= inv_r;
                acc[0] += s.ip_c[c] * inv_rp;
            } else {
                acc[0] += s.ip_c[c] * pow(r, -s.ip_p[c]);
            }
        }
    }
    block_sum<NT>(acc, v.red);
    if (threadIdx.x == 0) v.scal[S_ELI] = acc[1];
    return acc[0] + (s.ewald ? s.e_const : 0.0) + s.ip_tail;
}

// ───────────────────────── full evaluation ──────────────────────────────

template <int NT>
__device__ void evaluate_walker(const DevSys& s, const Smem& v, double* grec, const int2* pairs,
                                int npair) {
    const int np = s.np;
    // wrap every position into the cell (WalkerSet::load_all)
    for (int i = threadIdx.x; i < np; i += NT) {
        double r[3] = {v.pos[i * 2], v.pos[i * 2 + 1], 0.0};
        wrap_pos(s, r);
        v.pos[i * 2] = r[0];
        v.pos[i * 2 + 1] = r[1];
    }
    for (int i = threadIdx.x; i < np * 2; i += NT) {
        v.jg[i] = v.jl[i] = v.kg[i] = v.kl[i] = v.sg[i] = v.sl[i] = 0.0;
        if (s.cplx) v.pg[i] = v.pl[i] = 0.0;
    }
    if (threadIdx.x == 0) {
        v.scal[S_LOGPSI] = 0.0;
        v.scal[S_ERR] = 0.0;
        v.misc[M_ERR] = 0.0;
    }
    __syncthreads();
    double lp[1] = {0.0};
    // complex determinant: A = D⁻¹ from recomputed rows
    for (int b = 0; b < (s.cplx ? s.nblocks : 0); ++b) {
        c_gj_rebuild<NT>(s, v, b, -1, nullptr);
        if (threadIdx.x == 0) {
            double* bs = v.scal + S_BLOCK0 + 3 * b;
            bs[0] = v.misc[M_LOGDET];
            bs[1] = 0.0;
            bs[2] = 0.0;
            if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
            lp[0] += v.misc[M_LOGDET];
        }
        __syncthreads();
    }
    // backflow determinants: x, M, A = M⁻¹, F and every derivative
    if (s.nbf > 0) {
        bf_refresh_all<NT>(s, v, true);
        if (threadIdx.x == 0)
            for (int d = 0; d < s.nbf; ++d) lp[0] += v.scal[s.bf[d].oLS - s.o_scal];
        __syncthreads();
    }
    // determinants: rows, A = D⁻¹ by Gauss-Jordan, log|det|, condition
    for (int b = 0; b < (s.cplx ? 0 : s.nblocks); ++b) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n;
        double* D = grec + B.oD;
        double* Dg = grec + B.oDg;
        double* Dl = grec + B.oDl;
        double* rabs = v.scal - s.o_scal + B.orabs;
        for (int e = threadIdx.x; e < N * N; e += NT) {
            const int kr = e / N, m = e % N;
            double val, g[3], l[3];
            orbital(s, B, m, v.pos + (B.first + kr) * 2, val, g, l);
            D[e] = val;
            Dg[e * 2 + 0] = g[0];
            Dg[e * 2 + 1] = g[1];
            Dl[e * 2 + 0] = l[0];
            Dl[e * 2 + 1] = l[1];
        }
        __syncthreads();
        for (int kr = threadIdx.x; kr < N; kr += NT) {
            double sum = 0.0;
            for (int i = 0; i < N; ++i) sum += fabs(D[kr * N + i]);
            rabs[kr] = sum;
        }
        gj_rebuild<NT>(s, v, grec, b);
        double* A = v.scal - s.o_scal + B.oA;
        double ra = 0.0, rdm = 0.0;
        for (int a = threadIdx.x; a < N; a += NT) {
            double t = 0.0;
            for (int c = 0; c < N; ++c) t += fabs(A[a * N + c]);
            ra = fmax(ra, t);
            rdm = fmax(rdm, rabs[a]);
        }
        const double na = block_max<NT>(ra, v.red);
        const double nd = block_max<NT>(rdm, v.red);
        if (threadIdx.x == 0) {
            double* bs = v.scal + S_BLOCK0 + 3 * b;
            bs[0] = v.misc[M_LOGDET];
            bs[1] = 0.0;
            bs[2] = nd * na;
            if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
            lp[0] += v.misc[M_LOGDET];
        }
        __syncthreads();
    }
    // pair terms: each thread owns particle i and sums over its partners
    for (int i = threadIdx.x; i < np; i += NT) {
        double g[2] = {0.0, 0.0}, l[2] = {0.0, 0.0}, u_half = 0.0;
        for (int j = 0; j < np; ++j) {
            if (j == i) continue;
            double del[3];
            bool any = false;
            double r = 0.0;
            for (int t = 0; t < s.nterms; ++t) {
                const DevTerm& T = s.terms[t];
                if (!couples(T, i, j)) continue;
                if (!any) {
                    r = fold_dist(s, v.pos + i * 2, v.pos + j * 2, del);
                    any = true;
                }
                double u, du, d2u;
                radial(T, r, u, du, d2u);
                const double invr = 1.0 / r;
                u_half += 0.5 * u;
                for (int d = 0; d < 2; ++d) {
                    const double dor = del[d] * invr;
                    g[d] += du * dor;
                    l[d] += d2u * dor * dor + du * invr * (1.0 - dor * dor);
                }
            }
        }
        v.jg[i * 2] = g[0];
        v.jg[i * 2 + 1] = g[1];
        v.jl[i * 2] = l[0];
        v.jl[i * 2 + 1] = l[1];
        lp[0] += u_half;
    }
    // image sums: ρ per group from every particle's phases, then Σ w T
    if (s.nkJ > 0) {
        const int nk = s.nkJ;
        for (int e = threadIdx.x; e < s.ngroups * 2 * nk; e += NT) v.rho[e] = 0.0;
        const int m[2] = {s.m1J, s.m2J};
        for (int i = 0; i < np; ++i) {
            __syncthreads();
            const double th[2] = {s.recip[0] * v.pos[i * 2] + s.recip[1] * v.pos[i * 2 + 1],
                                  s.recip[2] * v.pos[i * 2] + s.recip[3] * v.pos[i * 2 + 1]};
            ladders<NT>(th, m, 2, v.lad);
            __syncthreads();
            double* rg = v.rho + s.group_of[i] * 2 * nk;
            for (int k = threadIdx.x; k < nk; k += NT) {
                double c, sn;
                phase_k(s, v.lad, v.lad + kLad, k, c, sn);
                rg[k] += c;
                rg[nk + k] += sn;
            }
        }
        __syncthreads();
        for (int t = 0; t < s.nterms; ++t) {
            const DevTerm& T = s.terms[t];
            if (!T.image) continue;
            const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
            const double* ar = v.rho + ga * 2 * nk;
            const double* br = v.rho + gb * 2 * nk;
            for (int k = threadIdx.x; k < nk; k += NT) {
                const double w = T.kw[k];
                lp[0] += T.same0 ? w * (ar[k] * ar[k] + ar[nk + k] * ar[nk + k])
                                 : 2.0 * w * (ar[k] * br[k] + ar[nk + k] * br[nk + k]);
            }
        }
    }
    block_sum<NT>(lp, v.red);
    __syncthreads();
    refresh_all<NT>(s, v, grec);
    const double el = local_energy<NT>(s, v, pairs, npair);
    if (threadIdx.x == 0) {
        v.scal[S_LOGPSI] = lp[0];
        v.scal[S_EL] = el;
    }
    __syncthreads();
}

}  // namespace

}  // namespace alea_gpu
