// Device-side system description, walker record layout and the per-walker
// math shared by the walker kernels (sm_100a).
//
// One CTA owns one walker for a whole sweep.  The walker's hot state (position,
// the gradient/Laplacian planes of the pair Jastrows, the k-space image sums
// and the determinants, the inverse matrices and the per-group structure
// factors ρ(k)) is staged from its HBM record into shared memory at kernel
// start and written back at the end; the orbital rows D, ∇D, ∇²D stay in HBM
// and are touched one row per move.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace alea_gpu {

constexpr int kMaxBlocks = 4;
constexpr int kMaxTerms = 8;
constexpr int kMaxGroups = 8;
constexpr int kMaxCoulomb = 8;
constexpr int kMaxN = 64;              // largest determinant block
constexpr int kMaxLadder = 16;         // largest |n| of a reciprocal index

// Scalar slots of a walker record.
enum : int {
    S_LOGPSI = 0, S_EL, S_WEIGHT, S_EPREV, S_RRP, S_RRA, S_AGE, S_ID, S_PARENT, S_ERR,
    S_NACC, S_NCUT, S_ELI /* Im E_L of a complex ψ */,
    S_BLOCK0 /* 3 per block: log|det|, updates, condition */,
    S_NSCAL = S_BLOCK0 + 3 * kMaxBlocks
};

struct DevSpline {
    double r_cut, inv_delta;
    int n_knots;
    const double* scaled;     // quintic Hermite data, 3 per knot (value, δ·f', δ²·f'')
    const double* poly;       // the same pieces as monomials in the local x: 6 per interval
};

struct DevTerm {
    int kind;                 // 0 Padé, 1 Drummond
    int npairs;
    int pairs[4][4];
    int nnum, nden;
    double coef[16];
    int image;
    DevSpline sp;
    double u_inf;
    const double* kw;         // weights on the shared Jastrow k set
    int same0;                // pairs[0] is a same-group pair
    int C;
    double gamma, L, alpha1;
    int ncoef;
    double dc[16];
    // kind 2, zero-energy: s = (p-2)/2, kappa, R_m, r_c, matching constants,
    // Chebyshev coefficients of sqrt(x) e^x K_{0,1}(x) in 4/x - 1 (2 x 24)
    double ze_s, ze_kappa, ze_rm, ze_rc, ze_c3, ze_logc1, ze_logc2;
    const double* ze_cheb;
};

// One optimisable parameter: a pair term's coefficient (alea_gpu_pair_term
// n_opt / opt_index: the term, which coefficient, and for an image-summed
// Padé the breakup of du/dp - inf, spline and k weights on the shared Jastrow
// k set), the shared width of a Gaussian orbital block (opt_alpha), or a
// backflow channel's parameter (kind 2: determinant `term`, channel `ch`,
// `index` the coefficient k of c_0..c_N or -1 for the cutoff L, `zs` set when
// the channel derives c_1 = C c_0 / L).
struct DevOpt {
    int kind;       // 0: a pair term's coefficient; 1: the shared width of Gaussian block `term`; 2: backflow
    int term;
    int index;
    int ch, zs;
    double inf;
    DevSpline sp;
    const double* kw;
};

struct DevBlock {
    int first, last, n, type;  // type 0 plane waves, 1 Gaussians, 2 twisted plane waves
    const double* k;          // plane waves [n*dim]; twisted: q = k + θ
    const double* is_sin;     // [n] (0/1)
    const double* centers;    // Gaussians [n*dim]
    const double* alphas;     // [n]
    int oA;                   // record offset of A (hot)
    int orabs;                // record offset of the row |D| sums (hot)
    long oD, oDg, oDl;        // record offsets of D, ∇D, ∇²D (cold)
};

struct DevBFCh {
    int sf, sl, C, nc;
    double L;
    double c[16];
};

// A backflow determinant: rows [first, last), orbitals, channels; offsets of
// its committed x, A, F, (log|det|, sign) in the hot record and of its
// pending copies (a proposal's) in the shared-memory scratch.
struct DevBF {
    int first, last, n, type;
    const double* k;
    const double* is_sin;
    const double* centers;
    const double* alphas;
    int nch;
    DevBFCh ch[4];
    int oX, oA, oF, oLS;
    int pX, pA, pF, pM;   // pM: log|det|', sign', g_x, g_y, valid
};

struct DevSys {
    int dim, np, periodic, ortho;
    double a[4], ainv[4], box[3], inv_box[3], cand[18], recip[4];
    int ngroups;
    int gfirst[kMaxGroups], glast[kMaxGroups];
    double gcharge[kMaxGroups];
    const double* inv_mass;   // [np*dim]
    const double* charge;     // [np]
    const int* group_of;      // [np]
    int nblocks, maxN;
    int cplx;                 // complex determinant (twisted plane waves): A = re | im
    DevBlock blocks[kMaxBlocks];
    int nterms;
    DevTerm terms[kMaxTerms];
    // bit t of gterms[ga][gb]: term t couples groups ga and gb (valid when
    // every term's pair ranges are whole groups, pair_by_group != 0)
    int pair_by_group;
    uint8_t gterms[kMaxGroups][kMaxGroups];
    // reciprocal vectors shared by every image-summed Jastrow term
    int nkJ, m1J, m2J;
    const int *n1J, *n2J;
    const double *kxJ, *kyJ, *kx2J, *ky2J;
    // Ewald
    int ewald;
    DevSpline esp;
    double e_rcut, e_inv_eps, e_const;
    int enk, e_m1, e_m2;
    const int *en1, *en2;
    const double* ew;
    int ncoul;
    int coul[kMaxCoulomb][4];
    double coul_coef[kMaxCoulomb];
    // inverse-power pair potentials C r^-p (integer p <= 16 by products, else pow)
    int nbf;
    DevBF bf[2];
    int nip;
    int ip[kMaxCoulomb][4];
    double ip_c[kMaxCoulomb], ip_p[kMaxCoulomb];
    int ip_pint[kMaxCoulomb];
    double ip_tail;
    // record layout (doubles): hot part [0, hot) is staged in shared memory
    long rec;                 // record stride
    int hot;
    int o_pos, o_jg, o_jl, o_kg, o_kl, o_sg, o_sl, o_scal, o_rho;
    int o_pg, o_pl;           // phase part of ∇ln ψ, ∂²ln ψ (complex determinant)
    // shared-memory scratch layout (doubles, after the hot part)
    int s_newpos, s_nval, s_ngrad, s_nlap, s_rad, s_cn, s_sn, s_co, s_so, s_col, s_rowp,
        s_red, s_misc, s_work, s_total;
    // shared-memory layout of the one-warp sweep (doubles; f_total = 0 when a
    // system does not take it): positions and pair-Jastrow planes, the record
    // from the scalars to the end of the hot part, the misc slots, then one
    // scratch area used by the moves (new orbital row, update vectors, and a
    // union of the partner and k-space changes with, in the FP32 form, the
    // FP64 rebuild's matrix) and, after the moves, by the local energy (sg,
    // sl, kg, kl planes and the k-space tables)
    int f_pos, f_jg, f_jl, f_scal, f_nval, f_ngrad, f_nlap, f_col, f_rowp, f_misc, f_work, f_cn,
        f_sn, f_co, f_so, f_sg, f_sl, f_kg, f_kl, f_elwork, f_total;
    int f_total32;            // the FP32 form's total: its FP64 rebuild needs N² in the move union
    int f32;                  // sweeps run the FP32 form (alea_gpu_set_precision)
    // three-dimensional walkers (alea_bf3d.cu): Ewald k-vectors [3*enk]
    // (kx, ky, kz per vector) and the shared-memory layout after the hot
    // part: proposal, misc slots, reduction area, pivot column, the pending
    // determinants of a proposal, then the move's work area (each
    // determinant's Gauss-Jordan multipliers and row exchanges; the moves'
    // layout ends there, at t_mtotal); the refresh's tables reuse the area
    // from the pending determinants on (t_work, up to t_total)
    const double* ek3;
    int t_newpos, t_misc, t_red, t_col, t_work, t_mwork, t_total;
    int t_mtotal;
    // ziggurat tables
    const uint64_t* zk;
    const double *zw, *zf;
    double zr;
};

// ───────────────────────── cell ─────────────────────────────────────────

__device__ __forceinline__ void min_image(const DevSys& s, double* del) {
    if (!s.periodic) return;
    if (s.ortho) {
        for (int d = 0; d < s.dim; ++d) del[d] = fma(-s.box[d], rint(del[d] * s.inv_box[d]), del[d]);
        return;
    }
    // General 2-D Bravais fold, in the operation order (and with the FMA
    // contraction) of the reference's fold_bravais_2d, branch-free select.
    double x0 = del[0], x1 = del[1];
    const double f0 = rint(fma(s.ainv[1], x1, s.ainv[0] * x0));
    const double f1 = rint(fma(s.ainv[3], x1, s.ainv[2] * x0));
    x0 -= fma(f1, s.a[2], f0 * s.a[0]);
    x1 -= fma(f1, s.a[3], f0 * s.a[1]);
    double b0 = x0, b1 = x1, best2 = fma(x1, x1, x0 * x0);
    for (int c = 1; c < 9; ++c) {
        const double y0 = x0 + s.cand[c * 2 + 0];
        const double y1 = x1 + s.cand[c * 2 + 1];
        const double r2 = fma(y1, y1, y0 * y0);
        const double take = (r2 < best2) ? 1.0 : 0.0;
        best2 = fma(take, r2 - best2, best2);
        b0 = fma(take, y0 - b0, b0);
        b1 = fma(take, y1 - b1, b1);
    }
    del[0] = b0;
    del[1] = b1;
}

__device__ __forceinline__ void wrap_pos(const DevSys& s, double* r) {
    if (!s.periodic) return;
    if (s.ortho) {
        for (int d = 0; d < s.dim; ++d) r[d] = fma(-s.box[d], rint(r[d] * s.inv_box[d]), r[d]);
        return;
    }
    const double f0 = rint(fma(s.ainv[1], r[1], s.ainv[0] * r[0]));
    const double f1 = rint(fma(s.ainv[3], r[1], s.ainv[2] * r[0]));
    r[0] -= fma(f1, s.a[2], f0 * s.a[0]);
    r[1] -= fma(f1, s.a[3], f0 * s.a[1]);
}

// Folded displacement xi - xj and its length.
__device__ __forceinline__ double fold_dist(const DevSys& s, const double* xi, const double* xj,
                                            double* del) {
    for (int d = 0; d < s.dim; ++d) del[d] = xi[d] - xj[d];
    min_image(s, del);
    double r2 = del[0] * del[0];
    for (int d = 1; d < s.dim; ++d) r2 = fma(del[d], del[d], r2);
    return sqrt(r2);
}

// 2-D forms of the above, same operation order, scalars instead of arrays.

__device__ __forceinline__ void min_image2(const DevSys& s, double& x0, double& x1) {
    if (!s.periodic) return;
    if (s.ortho) {
        x0 = fma(-s.box[0], rint(x0 * s.inv_box[0]), x0);
        x1 = fma(-s.box[1], rint(x1 * s.inv_box[1]), x1);
        return;
    }
    const double f0 = rint(fma(s.ainv[1], x1, s.ainv[0] * x0));
    const double f1 = rint(fma(s.ainv[3], x1, s.ainv[2] * x0));
    x0 -= fma(f1, s.a[2], f0 * s.a[0]);
    x1 -= fma(f1, s.a[3], f0 * s.a[1]);
    double b0 = x0, b1 = x1, best2 = fma(x1, x1, x0 * x0);
#pragma unroll
    for (int c = 1; c < 9; ++c) {
        const double y0 = x0 + s.cand[c * 2 + 0];
        const double y1 = x1 + s.cand[c * 2 + 1];
        const double r2 = fma(y1, y1, y0 * y0);
        const double take = (r2 < best2) ? 1.0 : 0.0;
        best2 = fma(take, r2 - best2, best2);
        b0 = fma(take, y0 - b0, b0);
        b1 = fma(take, y1 - b1, b1);
    }
    x0 = b0;
    x1 = b1;
}

// Folded displacement a - b and its length.
__device__ __forceinline__ double fold2(const DevSys& s, double ax, double ay, double bx, double by,
                                        double& dx, double& dy) {
    dx = ax - bx;
    dy = ay - by;
    min_image2(s, dx, dy);
    return sqrt(fma(dy, dy, dx * dx));
}

__device__ __forceinline__ void wrap2(const DevSys& s, double& x, double& y) {
    if (!s.periodic) return;
    if (s.ortho) {
        x = fma(-s.box[0], rint(x * s.inv_box[0]), x);
        y = fma(-s.box[1], rint(y * s.inv_box[1]), y);
        return;
    }
    const double f0 = rint(fma(s.ainv[1], y, s.ainv[0] * x));
    const double f1 = rint(fma(s.ainv[3], y, s.ainv[2] * x));
    x -= fma(f1, s.a[2], f0 * s.a[0]);
    y -= fma(f1, s.a[3], f0 * s.a[1]);
}

// ───────────────────────── radial functions ─────────────────────────────

// Read-only table loads that ask L1 to keep the line (evict_last): the
// spline, k-vector and weight tables are shared by every walker on an SM,
// while the walker records stream through.
__device__ __forceinline__ double2 ldg_keep(const double2* p) {
    double2 r;
    asm("ld.global.nc.L1::evict_last.v2.f64 {%0, %1}, [%2];" : "=d"(r.x), "=d"(r.y) : "l"(p));
    return r;
}

__device__ __forceinline__ double ldg_keep(const double* p) {
    double r;
    asm("ld.global.nc.L1::evict_last.f64 %0, [%1];" : "=d"(r) : "l"(p));
    return r;
}

// The breakup's quintic Hermite spline, evaluated from its per-interval
// monomial form c_0 + c_1 x + ... + c_5 x^5 in the local coordinate
// x = r/δ - i (the host expands each interval's Hermite data once).
__device__ __forceinline__ void spline3(const DevSpline& sp, double r, double& f, double& df,
                                        double& d2f) {
    if (r >= sp.r_cut) {
        f = df = d2f = 0.0;
        return;
    }
    const double t = r * sp.inv_delta;
    int i = static_cast<int>(t);
    if (i > sp.n_knots - 2) i = sp.n_knots - 2;
    const double x = t - i;
    const double2* c2 = reinterpret_cast<const double2*>(sp.poly + 6 * i);
    const double2 c01 = ldg_keep(c2), c23 = ldg_keep(c2 + 1), c45 = ldg_keep(c2 + 2);
    f = fma(fma(fma(fma(fma(c45.y, x, c45.x), x, c23.y), x, c23.x), x, c01.y), x, c01.x);
    const double g = fma(fma(fma(fma(5.0 * c45.y, x, 4.0 * c45.x), x, 3.0 * c23.y), x, 2.0 * c23.x), x, c01.y);
    const double h = fma(fma(fma(20.0 * c45.y, x, 12.0 * c45.x), x, 6.0 * c23.y), x, 2.0 * c23.x);
    df = sp.inv_delta * g;
    d2f = sp.inv_delta * sp.inv_delta * h;
}

__device__ __forceinline__ double spline1(const DevSpline& sp, double r) {
    if (r >= sp.r_cut) return 0.0;
    const double t = r * sp.inv_delta;
    int i = static_cast<int>(t);
    if (i > sp.n_knots - 2) i = sp.n_knots - 2;
    const double x = t - i;
    const double2* c2 = reinterpret_cast<const double2*>(sp.poly + 6 * i);
    const double2 c01 = ldg_keep(c2), c23 = ldg_keep(c2 + 1), c45 = ldg_keep(c2 + 2);
    return fma(fma(fma(fma(fma(c45.y, x, c45.x), x, c23.y), x, c23.x), x, c01.y), x, c01.x);
}

__device__ __forceinline__ void poly_acc(const double* c, int n, double r, double& v, double& dv,
                                         double& d2v) {
    double r_km1 = 1.0, r_km2 = 0.0;
    for (int i = 0; i < n; ++i) {
        const int k = i + 1;
        v += c[i] * r_km1 * r;
        dv += c[i] * k * r_km1;
        d2v += c[i] * k * (k - 1) * r_km2;
        r_km2 = r_km1;
        r_km1 *= r;
    }
}

// e^x K0(x) and e^x K1(x), x > 0: the ascending series for x <= 2 (DLMF
// 10.31.1-2, 15 terms), else the Chebyshev series of sqrt(x) e^x K_nu(x) in
// ξ = 4/x - 1 summed by Clenshaw's recurrence (24 terms per order).
__device__ __forceinline__ void bessel_k01e(const double* cheb, double x, double& k0e, double& k1e) {
    if (x <= 2.0) {
        const double euler_gamma = 0.57721566490153286060651209008240243;
        const double y = 0.25 * x * x;
        double term0 = 1.0, term1 = 1.0, harmonic = 0.0;
        double i0 = 0.0, s0 = 0.0, i1 = 0.0, s1 = 0.0;
        for (int k = 0; k < 15; ++k) {
            if (k > 0) {
                term0 *= y / (static_cast<double>(k) * k);
                term1 *= y / (static_cast<double>(k) * (k + 1));
                harmonic += 1.0 / k;
            }
            const double harmonic_next = harmonic + 1.0 / (k + 1);
            i0 += term0;
            s0 += harmonic * term0;
            i1 += term1;
            s1 += (harmonic + harmonic_next - 2.0 * euler_gamma) * term1;
        }
        const double lh = log(0.5 * x);
        const double k0 = -(lh + euler_gamma) * i0 + s0;
        const double k1 = 1.0 / x + lh * (0.5 * x * i1) - 0.25 * x * s1;
        const double ex = exp(x);
        k0e = ex * k0;
        k1e = ex * k1;
        return;
    }
    const double xi = 4.0 / x - 1.0, two_xi = 2.0 * xi;
    double b0 = 0.0, b0p = 0.0, b1 = 0.0, b1p = 0.0;
    for (int k = 23; k >= 1; --k) {
        const double t0 = two_xi * b0 - b0p + __ldg(cheb + k);
        const double t1 = two_xi * b1 - b1p + __ldg(cheb + 24 + k);
        b0p = b0;
        b0 = t0;
        b1p = b1;
        b1 = t1;
    }
    const double isx = 1.0 / sqrt(x);
    k0e = (xi * b0 - b0p + __ldg(cheb)) * isx;
    k1e = (xi * b1 - b1p + __ldg(cheb + 24)) * isx;
}

// u, u', u'' of the zero-energy Jastrow at r (kind 2 below), out of line:
// its Bessel series are long and rarely on the path of a move.
static __device__ __noinline__ void radial_zero_energy(double r, double ze_s, double ze_kappa, double ze_rm,
                                                double ze_rc, double ze_c3, double ze_logc1,
                                                double ze_logc2, const double* ze_cheb, double& u,
                                                double& du, double& d2u) {
    if (r < ze_rm) {   // ln[C1 K0(κ r^-s)]; s = 1/2 (1/r³ dipoles) without pow
        const double x = ze_kappa * (ze_s == 0.5 ? 1.0 / sqrt(r) : pow(r, -ze_s));
        double k0e, k1e;
        bessel_k01e(ze_cheb, x, k0e, k1e);
        const double q = k1e / k0e;
        const double sx = ze_s * x;
        u = log(k0e) - x + ze_logc1;
        du = sx * q / r;
        d2u = sx / (r * r) * (sx * (1.0 - q) * (1.0 + q) - q);
        return;
    }
    const double rr = fmin(r, ze_rc);
    const double inv_r = 1.0 / rr;
    const double inv_c = 1.0 / (2.0 * ze_rc - rr);
    const double m = (r < ze_rc) ? 1.0 : 0.0;
    const double a = ze_c3;
    u = m * (ze_logc2 - a * inv_r - a * inv_c);
    du = m * (a * inv_r * inv_r - a * inv_c * inv_c);
    d2u = m * (-2.0 * a * inv_r * inv_r * inv_r - 2.0 * a * inv_c * inv_c * inv_c);
}

// u, u', u'' of a Padé (kind 0) or Drummond (kind 1) pair term at r (the
// short-range half for an image sum).
__device__ __forceinline__ void radial_pd(const DevTerm& T, double r, double& u, double& du,
                                          double& d2u) {
    if (T.kind == 0) {
        double p = 0.0, dp = 0.0, d2p = 0.0;
        double q = 1.0, dq = 0.0, d2q = 0.0;
        if (T.nnum == 1 && T.nden == 1) {   // a r / (1 + b r): the sums below, unrolled
            const double a = T.coef[0], b = T.coef[1];
            p = a * r;
            dp = a;
            q = fma(b, r, 1.0);
            dq = b;
        } else {
            poly_acc(T.coef, T.nnum, r, p, dp, d2p);
            poly_acc(T.coef + T.nnum, T.nden, r, q, dq, d2q);
        }
        const double inv_q = 1.0 / q;
        u = p * inv_q;
        du = (dp * q - p * dq) * inv_q * inv_q;
        d2u = (d2p - (2.0 * dp * dq - 2.0 * p * dq * dq * inv_q + p * d2q) * inv_q) * inv_q;
        if (T.image) {
            if (r >= T.sp.r_cut) {
                u = du = d2u = 0.0;
                return;
            }
            double f, df, d2f;
            spline3(T.sp, r, f, df, d2f);
            u -= T.u_inf + f;
            du -= df;
            d2u -= d2f;
        }
        return;
    }
    const double t = r - T.L;
    double tCm2 = 1.0;
    for (int i = 0; i < T.C - 2; ++i) tCm2 *= t;
    const double tCm1 = tCm2 * t, tC = tCm1 * t;
    const double g = tC, dg = static_cast<double>(T.C) * tCm1,
                 d2g = static_cast<double>(T.C) * (T.C - 1) * tCm2;
    double P = T.dc[0] + T.alpha1 * r, dP = T.alpha1, d2P = 0.0;
    double r_lm2 = 1.0, r_lm1 = r, r_l = r * r;
    for (int k = 1; k < T.ncoef; ++k) {
        const int l = k + 1;
        const double c = T.dc[k];
        P += c * r_l;
        dP += c * l * r_lm1;
        d2P += c * l * (l - 1) * r_lm2;
        r_lm2 = r_lm1;
        r_lm1 = r_l;
        r_l *= r;
    }
    const double m = (r < T.L) ? 1.0 : 0.0;
    u = m * (g * P);
    du = m * (dg * P + g * dP);
    d2u = m * (d2g * P + 2.0 * dg * dP + g * d2P);
}

// u, u', u'' of any pair term at r.
__device__ __forceinline__ void radial(const DevTerm& T, double r, double& u, double& du,
                                       double& d2u) {
    if (T.kind == 2) {
        if (r >= T.ze_rm) {   // the tail, inline (the Bessel form below r_m is the rare call)
            const double rr = fmin(r, T.ze_rc);
            const double inv_r = 1.0 / rr;
            const double inv_c = 1.0 / (2.0 * T.ze_rc - rr);
            const double m = (r < T.ze_rc) ? 1.0 : 0.0;
            const double a = T.ze_c3;
            u = m * (T.ze_logc2 - a * inv_r - a * inv_c);
            du = m * (a * inv_r * inv_r - a * inv_c * inv_c);
            d2u = m * (-2.0 * a * inv_r * inv_r * inv_r - 2.0 * a * inv_c * inv_c * inv_c);
            return;
        }
        radial_zero_energy(r, T.ze_s, T.ze_kappa, T.ze_rm, T.ze_rc, T.ze_c3, T.ze_logc1, T.ze_logc2,
                           T.ze_cheb, u, du, d2u);
        return;
    }
    radial_pd(T, r, u, du, d2u);
}

// Does term T couple particles p and k (any of its group pairs)?
__device__ __forceinline__ bool couples(const DevTerm& T, int p, int k) {
    for (int q = 0; q < T.npairs; ++q) {
        const int af = T.pairs[q][0], al = T.pairs[q][1], bf = T.pairs[q][2], bl = T.pairs[q][3];
        const bool pa = p >= af && p < al, pb = p >= bf && p < bl;
        const bool ka = k >= af && k < al, kb = k >= bf && k < bl;
        if (af == bf && al == bl) {
            if (pa && ka && p != k) return true;
        } else if ((pa && kb) || (pb && ka)) {
            return true;
        }
    }
    return false;
}

// Bit mask of the terms coupling particles p and k.
__device__ __forceinline__ unsigned coupling(const DevSys& s, int p, int k) {
    if (s.pair_by_group) return s.gterms[s.group_of[p]][s.group_of[k]];
    unsigned m = 0;
    for (int t = 0; t < s.nterms; ++t)
        if (couples(s.terms[t], p, k)) m |= 1u << t;
    return m;
}

__device__ __forceinline__ bool in_term(const DevTerm& T, int p) {
    for (int q = 0; q < T.npairs; ++q)
        if ((p >= T.pairs[q][0] && p < T.pairs[q][1]) || (p >= T.pairs[q][2] && p < T.pairs[q][3]))
            return true;
    return false;
}

// ───────────────────────── orbitals ─────────────────────────────────────

// Orbital i of block B at position r: value, gradient[dim], Laplacian[dim].
__device__ __forceinline__ void orbital(const DevSys& s, const DevBlock& B, int i, const double* r,
                                        double& val, double* grad, double* lap) {
    const int dim = s.dim;
    if (B.type == 0) {
        const double* ki = B.k + i * dim;
        double phase = 0.0;
        for (int d = 0; d < dim; ++d) phase += ki[d] * r[d];
        double sn, c;
        sincos(phase, &sn, &c);
        if (B.is_sin[i] != 0.0) {
            val = sn;
            for (int d = 0; d < dim; ++d) {
                grad[d] = ki[d] * c;
                lap[d] = -ki[d] * ki[d] * sn;
            }
        } else {
            val = c;
            for (int d = 0; d < dim; ++d) {
                grad[d] = -ki[d] * sn;
                lap[d] = -ki[d] * ki[d] * c;
            }
        }
    } else {
        const double alpha = B.alphas[i];
        double del[3];
        for (int d = 0; d < dim; ++d) del[d] = r[d] - B.centers[i * dim + d];
        min_image(s, del);
        double r2 = 0.0;
        for (int d = 0; d < dim; ++d) r2 += del[d] * del[d];
        const double phi = exp(-alpha * r2);
        val = phi;
        for (int d = 0; d < dim; ++d) {
            grad[d] = phi * (-2.0 * alpha * del[d]);
            lap[d] = phi * (4.0 * alpha * alpha * del[d] * del[d] - 2.0 * alpha);
        }
    }
}

// ───────────────────────── reductions ───────────────────────────────────

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K values over the CTA of NT threads; every thread gets the totals.  A
// one-warp CTA uses shuffles only; wider ones go through `red`
// (NT/32*K + K doubles) with two barriers.
template <int NT, int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red) {
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] = warp_sum(v[k]);
    if constexpr (NT > 32) {
        constexpr int W = NT / 32;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < K; ++k) red[warp * K + k] = v[k];
        __syncthreads();
        if (threadIdx.x < K) {
            double t = 0.0;
            for (int w = 0; w < W; ++w) t += red[w * K + threadIdx.x];
            red[W * K + threadIdx.x] = t;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = red[W * K + k];
        __syncthreads();
    }
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if constexpr (NT > 32) {
        constexpr int W = NT / 32;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        if (lane == 0) red[warp] = v;
        __syncthreads();
        double m = red[0];
        for (int w = 1; w < W; ++w) m = fmax(m, red[w]);
        __syncthreads();
        return m;
    }
    return v;
}

// ───────────────────────── random numbers ───────────────────────────────

struct Xo {
    uint64_t s0, s1, s2, s3;
};

__device__ __forceinline__ uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

__device__ __forceinline__ uint64_t xo_next(Xo& r) {
    const uint64_t result = rotl64(r.s0 + r.s3, 23) + r.s0;
    const uint64_t t = r.s1 << 17;
    r.s2 ^= r.s0;
    r.s3 ^= r.s1;
    r.s1 ^= r.s2;
    r.s0 ^= r.s3;
    r.s2 ^= t;
    r.s3 = rotl64(r.s3, 45);
    return result;
}

__device__ __forceinline__ double xo_uniform(Xo& r) {
    return static_cast<double>(static_cast<int64_t>(xo_next(r) >> 11)) * 0x1.0p-53;
}

// Ziggurat normal deviate with the region/sign/position split of the
// reference's XoshiroRandom::gaussian.
__device__ __forceinline__ double xo_gaussian(Xo& r, const uint64_t* zk, const double* zw,
                                              const double* zf, double zr) {
    for (int guard = 0; guard < 1 << 20; ++guard) {
        const uint64_t bits = xo_next(r);
        const unsigned i = static_cast<unsigned>(bits & 0xff);
        const uint64_t sign = (bits & 0x100) << 55;
        const uint64_t position = (bits >> 9) & ((uint64_t{1} << 52) - 1);
        const double x = static_cast<double>(static_cast<int64_t>(position)) * zw[i];
        if (position < zk[i]) return __longlong_as_double(__double_as_longlong(x) ^ sign);
        if (i == 0) {
            for (int g2 = 0; g2 < 1 << 20; ++g2) {
                const double xi = -log1p(-xo_uniform(r)) / zr;
                const double y = -log1p(-xo_uniform(r));
                if (y + y > xi * xi)
                    return __longlong_as_double(__double_as_longlong(zr + xi) ^ sign);
            }
            return 0.0;
        }
        if (zf[i] + xo_uniform(r) * (zf[i - 1] - zf[i]) < exp(-0.5 * x * x))
            return __longlong_as_double(__double_as_longlong(x) ^ sign);
    }
    return 0.0;
}

}  // namespace alea_gpu
