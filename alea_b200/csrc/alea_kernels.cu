// Walker kernels for sm_100a: full evaluation, the fused VMC/DMC sweep for
// CTAs of 32, 64 or 128 threads, single moves for the component-level ABI,
// the per-stream random-number draw and the branching gather.  The device
// functions they call are in alea_walker.cuh.
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "alea_walker.cuh"

namespace alea_gpu {

// ───────────────────────── kernels ──────────────────────────────────────

template <int NT>
__global__ void __launch_bounds__(NT) evaluate_kernel(DevSys s, double* records, int nw,
                                                      const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_hot<NT>(s, rec, sm);
    const Smem v = view(s, sm);
    evaluate_walker<NT>(s, v, rec, pairs, npair);
    store_hot<NT>(s, rec, sm);
}

// d u / d p of parameter `o` of its term at pair distance r: Padé
// du/da_k = r^k / Q, du/db_k = -P r^k / Q^2 (pade_jastrow.cpp:208-213);
// Drummond u = (r - L)^C (alpha_0 + alpha_1 r + sum_l alpha_l r^l) below L with
// alpha_1 = Gamma / (-L)^C + alpha_0 C / L (drummond_jastrow.cpp:201-320).
__device__ double dudp(const DevTerm& T, const DevOpt& o, double r) {
    if (T.kind == 0) {
        double P = 0.0, Q = 1.0, rk = 1.0;
        for (int k = 0; k < T.nnum; ++k) {
            rk *= r;
            P = fma(T.coef[k], rk, P);
        }
        rk = 1.0;
        for (int k = 0; k < T.nden; ++k) {
            rk *= r;
            Q = fma(T.coef[T.nnum + k], rk, Q);
        }
        if (o.index < T.nnum) {
            double rp = 1.0;
            for (int k = 0; k <= o.index; ++k) rp *= r;
            return rp / Q;
        }
        double rp = 1.0;
        for (int k = 0; k <= o.index - T.nnum; ++k) rp *= r;
        return -P * rp / (Q * Q);
    }
    // Drummond
    if (r >= T.L) return 0.0;
    const double d = r - T.L;
    double g = 1.0;   // (r - L)^C
    for (int i = 0; i < T.C; ++i) g *= d;
    const double C = static_cast<double>(T.C);
    if (o.index == 0) return g * fma(C / T.L, r, 1.0);
    if (o.index < T.ncoef) {
        double rp = 1.0;
        for (int k = 0; k <= o.index; ++k) rp *= r;   // alpha_{index+1} r^{index+1}
        return g * rp;
    }
    // the cutoff L: d/dL of (r - L)^C P(r) with alpha_1(L)
    double P = T.dc[0] + T.alpha1 * r, rp = r;
    for (int k = 1; k < T.ncoef; ++k) {
        rp *= r;
        P = fma(T.dc[k], rp, P);
    }
    double gm1 = 1.0;
    for (int i = 0; i + 1 < T.C; ++i) gm1 *= d;
    double ipw = 1.0;
    for (int i = 0; i < T.C + 1; ++i) ipw *= -T.L;
    const double dalpha1 = T.gamma * C / ipw - T.dc[0] * C / (T.L * T.L);
    return -C * gm1 * P + g * dalpha1 * r;
}

// d u / d p with its first and second r-derivatives (the same functions as
// dudp): Padé by the quotient rule on N/D (N = r^k, D = Q for a_k;
// N = -P r^k, D = Q^2 for b_k); Drummond by the product rule on
// (r - L)^m times a polynomial.  Zero for a Drummond pair beyond L.
__device__ void dudp3(const DevTerm& T, const DevOpt& o, double r, double& v, double& d1, double& d2) {
    auto powi = [](double x, int n) {
        double y = 1.0;
        for (int i = 0; i < n; ++i) y *= x;
        return n < 0 ? 0.0 : y;
    };
    if (T.kind == 0) {
        double P = 0.0, P1 = 0.0, P2 = 0.0, Q = 1.0, Q1 = 0.0, Q2 = 0.0;
        for (int k = 1; k <= T.nnum; ++k) {
            const double a = T.coef[k - 1];
            P += a * powi(r, k);
            P1 += a * k * powi(r, k - 1);
            P2 += a * k * (k - 1) * powi(r, k - 2);
        }
        for (int k = 1; k <= T.nden; ++k) {
            const double b = T.coef[T.nnum + k - 1];
            Q += b * powi(r, k);
            Q1 += b * k * powi(r, k - 1);
            Q2 += b * k * (k - 1) * powi(r, k - 2);
        }
        double N, N1, N2, D, D1, D2;
        if (o.index < T.nnum) {
            const int k = o.index + 1;
            N = powi(r, k);
            N1 = k * powi(r, k - 1);
            N2 = k * (k - 1) * powi(r, k - 2);
            D = Q;
            D1 = Q1;
            D2 = Q2;
        } else {
            const int k = o.index - T.nnum + 1;
            const double rk = powi(r, k), rk1 = k * powi(r, k - 1), rk2 = k * (k - 1) * powi(r, k - 2);
            N = -P * rk;
            N1 = -(P1 * rk + P * rk1);
            N2 = -(P2 * rk + 2.0 * P1 * rk1 + P * rk2);
            D = Q * Q;
            D1 = 2.0 * Q * Q1;
            D2 = 2.0 * (Q1 * Q1 + Q * Q2);
        }
        v = N / D;
        d1 = (N1 - v * D1) / D;
        d2 = (N2 - 2.0 * d1 * D1 - v * D2) / D;
        return;
    }
    v = d1 = d2 = 0.0;
    if (r >= T.L) return;
    const int C = T.C;
    const double x = r - T.L;
    // (r - L)^m and its two r-derivatives
    auto g = [&](int m, double& g0, double& g1, double& g2) {
        g0 = powi(x, m);
        g1 = m * powi(x, m - 1);
        g2 = m * (m - 1) * powi(x, m - 2);
    };
    auto product = [&](double a0, double a1, double a2, double b0, double b1, double b2, double s) {
        v += s * a0 * b0;
        d1 += s * (a1 * b0 + a0 * b1);
        d2 += s * (a2 * b0 + 2.0 * a1 * b1 + a0 * b2);
    };
    double g0, g1, g2;
    g(C, g0, g1, g2);
    if (o.index == 0) {   // alpha_0, with alpha_1's dependence C / L
        product(g0, g1, g2, 1.0 + C / T.L * r, C / T.L, 0.0, 1.0);
        return;
    }
    if (o.index < T.ncoef) {   // alpha_l r^l, l = index + 1
        const int l = o.index + 1;
        product(g0, g1, g2, powi(r, l), l * powi(r, l - 1), l * (l - 1) * powi(r, l - 2), 1.0);
        return;
    }
    // the cutoff L: -C (r - L)^{C-1} P(r) + (r - L)^C (d alpha_1 / dL) r
    double P = T.dc[0] + T.alpha1 * r, P1 = T.alpha1, P2 = 0.0;
    for (int k = 1; k < T.ncoef; ++k) {
        const int l = k + 1;
        P += T.dc[k] * powi(r, l);
        P1 += T.dc[k] * l * powi(r, l - 1);
        P2 += T.dc[k] * l * (l - 1) * powi(r, l - 2);
    }
    double h0, h1, h2;
    g(C - 1, h0, h1, h2);
    product(h0, h1, h2, P, P1, P2, -static_cast<double>(C));
    const double ipw = powi(-T.L, C + 1);
    const double dalpha1 = T.gamma * C / ipw - T.dc[0] * C / (T.L * T.L);
    product(g0, g1, g2, r, 1.0, 0.0, dalpha1);
}

// d(grad ln psi)/dp_q and d(lap ln psi)/dp_q for one walker, each particle
// on its own thread summing over its partners in the parameter's term
// (PadeJastrow / DrummondJastrow::compute_parameter_gradient_derivatives,
// pade_jastrow.cpp:806-880): with f1, f2 the r-derivatives of du/dp (minus the
// image sum's long-range part inside r_cut), grad += f1 Δ/r and
// lap += f2 (Δ/r)^2 + f1 (1 - (Δ/r)^2) / r; the image sum's k-space part
// (kspace_pair_sum.cpp:91-107, :315-320) from the particle's phases and the
// other side's rho(k).  Outputs [q][p*2 + d][nw]; other particles untouched.
template <int NT>
__global__ void __launch_bounds__(NT) param_grad_kernel(DevSys s, const double* records, int nw,
                                                        const DevOpt* opts, int nopt, double* dgrad,
                                                        double* dlap) {
    __shared__ double pos[2 * 256];
    const int w = blockIdx.x;
    if (w >= nw || s.np > 256) return;
    const double* rec = records + static_cast<long>(w) * s.rec;
    for (int i = threadIdx.x; i < s.np * 2; i += NT) pos[i] = rec[s.o_pos + i];
    __syncthreads();
    const long plane = static_cast<long>(s.np) * 2 * nw;
    for (int q = 0; q < nopt; ++q) {
        const DevOpt& o = opts[q];
        if (o.kind != 0) continue;   // orbital widths: orbital_param_kernel
        const DevTerm& T = s.terms[o.term];
        for (int i = threadIdx.x; i < s.np; i += NT) {
            double gx = 0.0, gy = 0.0, lx = 0.0, ly = 0.0;
            bool touched = false;
            for (int pp = 0; pp < T.npairs; ++pp) {
                const int af = T.pairs[pp][0], al = T.pairs[pp][1], bf = T.pairs[pp][2], bl = T.pairs[pp][3];
                const bool same = af == bf && al == bl;
                const bool in_a = i >= af && i < al, in_b = i >= bf && i < bl;
                for (int side = 0; side < 2; ++side) {
                    if (side == 0 ? !in_a : (same || !in_b)) continue;
                    touched = true;
                    const int jf = side == 0 ? bf : af, jl = side == 0 ? bl : al;
                    for (int j = jf; j < jl; ++j) {
                        if (j == i) continue;
                        double del[3];
                        const double r = fold_dist(s, pos + i * 2, pos + j * 2, del);
                        double v, f1, f2;
                        dudp3(T, o, r, v, f1, f2);
                        if (T.image) {
                            if (r >= o.sp.r_cut) continue;
                            double f, df, d2f;
                            spline3(o.sp, r, f, df, d2f);
                            f1 -= df;
                            f2 -= d2f;
                        }
                        const double inv_r = 1.0 / r;
                        const double ox = del[0] * inv_r, oy = del[1] * inv_r;
                        gx += f1 * ox;
                        gy += f1 * oy;
                        lx += f2 * ox * ox + f1 * inv_r * (1.0 - ox * ox);
                        ly += f2 * oy * oy + f1 * inv_r * (1.0 - oy * oy);
                    }
                }
            }
            if (T.image && touched) {
                const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
                const bool in_a = i >= T.pairs[0][0] && i < T.pairs[0][1];
                const int go = T.same0 ? ga : (in_a ? gb : ga);
                const double self = T.same0 ? 1.0 : 0.0;
                const double* pr = rec + s.o_rho + 2 * go * s.nkJ;
                const double* pi = pr + s.nkJ;
                const double x = pos[i * 2], y = pos[i * 2 + 1];
                for (int k = 0; k < s.nkJ; ++k) {
                    double sn, c;
                    sincos(s.kxJ[k] * x + s.kyJ[k] * y, &sn, &c);
                    const double gk = 2.0 * o.kw[k] * (c * pi[k] - sn * pr[k]);
                    const double lk = 2.0 * o.kw[k] * (self - (c * pr[k] + sn * pi[k]));
                    gx += s.kxJ[k] * gk;
                    gy += s.kyJ[k] * gk;
                    lx += s.kx2J[k] * lk;
                    ly += s.ky2J[k] * lk;
                }
            }
            if (!touched) continue;
            const long base = q * plane + static_cast<long>(i) * 2 * nw + w;
            dgrad[base] = gx;
            dgrad[base + nw] = gy;
            dlap[base] = lx;
            dlap[base + nw] = ly;
        }
    }
}

// O_q = d ln psi / d p_q of every optimisable parameter for one walker: the
// ∂η/∂p at r of one backflow parameter (BackflowFunction::parameter_derivatives,
// backflow_function.h:111-135): k >= 0 the coefficient c_k, ∂η/∂c_k = f r^k
// with f = (1 - r/L)^C (plus f C r/L for c_0 when c_1 = C c_0/L, zs); k = -1
// the cutoff, ∂η/∂L = C t^{C-1} r/L² P(r) (minus f C c_0 r/L² when zs).
__device__ __forceinline__ double bf_eta_dparam(const DevBFCh& C, int k, int zs, double r) {
    if (r >= C.L) return 0.0;
    const double t = 1.0 - r / C.L;
    double tc1 = 1.0;
    for (int i = 0; i < C.C - 1; ++i) tc1 *= t;
    const double f = tc1 * t;
    if (k >= 0) {
        double rk = 1.0;
        for (int i = 0; i < k; ++i) rk *= r;
        double v = f * rk;
        if (zs && k == 0) v += f * static_cast<double>(C.C) * r / C.L;
        return v;
    }
    double P = 0.0;
    for (int i = C.nc - 1; i >= 0; --i) P = P * r + C.c[i];
    double v = static_cast<double>(C.C) * tc1 * r / (C.L * C.L) * P;
    if (zs) v -= f * static_cast<double>(C.C) * C.c[0] * r / (C.L * C.L);
    return v;
}

// ∂η/∂p, ∂η'/∂p and ∂η''/∂p at r of one backflow parameter (k >= 0 the
// coefficient c_k, k = -1 the cutoff; zs: c_1 = C c_0/L), zero beyond L
// (BackflowFunction::parameter_derivatives, backflow_function.h:137-196;
// the channel's truncation C >= 3).  With t = 1 - r/L and f = t^C, a
// coefficient multiplies b(r) = r^k (plus C r/L for c_0 when zs):
// (f b, f'b + f b', f''b + 2f'b' + f b'').  The cutoff moves f by
// g = ∂f/∂L = (C/L²) r t^{C-1} and, when zs, c_1 by a = -C c_0/L².
__device__ void bf_eta_dparam3(const DevBFCh& C, int k, int zs, double r, double& de, double& d1, double& d2) {
    de = d1 = d2 = 0.0;
    if (r >= C.L) return;
    const double Cd = static_cast<double>(C.C), L = C.L;
    const double t = 1.0 - r / L;
    double tc3 = 1.0;
    for (int i = 0; i < C.C - 3; ++i) tc3 *= t;
    const double tc2 = tc3 * t, tc1 = tc2 * t, f = tc1 * t;
    const double fp = -Cd / L * tc1, fpp = Cd * (Cd - 1.0) / (L * L) * tc2;
    if (k >= 0) {
        double b = 1.0, b1 = 0.0, b2 = 0.0;   // r^k, k r^{k-1}, k(k-1) r^{k-2}
        for (int i = 0; i < k; ++i) {
            b2 = b2 * r + 2.0 * b1;
            b1 = b1 * r + b;
            b *= r;
        }
        if (zs && k == 0) {
            b += Cd * r / L;
            b1 += Cd / L;
        }
        de = f * b;
        d1 = fp * b + f * b1;
        d2 = fpp * b + 2.0 * fp * b1 + f * b2;
        return;
    }
    double P = 0.0, Pp = 0.0, Ppp = 0.0;
    for (int i = C.nc - 1; i >= 0; --i) {
        Ppp = Ppp * r + 2.0 * Pp;
        Pp = Pp * r + P;
        P = P * r + C.c[i];
    }
    const double pre = Cd / (L * L);
    const double g = pre * r * tc1;
    const double g1 = pre * (tc1 - (Cd - 1.0) * (r / L) * tc2);
    const double g2 = Cd * (Cd - 1.0) / (L * L * L) * (-2.0 * tc2 + (Cd - 2.0) * (r / L) * tc3);
    const double a = zs ? -Cd * C.c[0] / (L * L) : 0.0;
    de = g * P + f * a * r;
    d1 = g1 * P + g * Pp + fp * a * r + f * a;
    d2 = g2 * P + 2.0 * g1 * Pp + g * Ppp + fpp * a * r + 2.0 * fp * a;
}

// The pair tensors B = e δ + e1 r̂ r̂ᵀ r and S_{αβ} = ∂²_β [e r_α] of a radial
// function with values (e, e1, e2) at the displacement del (|del| = r > 0):
// the same forms as bf_pair's, here for the parameter derivative of η.
__device__ __forceinline__ void bf_tensors(double e, double e1, double e2, const double* del, double r, double* B,
                                           double* S) {
    const double inv_r = r > 0.0 ? 1.0 / r : 0.0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            B[a * 2 + b] = (a == b ? e : 0.0) + e1 * del[a] * del[b] * inv_r;
            const double rb2 = del[b] * del[b] * inv_r * inv_r;
            S[a * 2 + b] = (a == b ? 2.0 * e1 * del[b] * inv_r : 0.0) + del[a] * (e2 * rb2 + e1 * inv_r * (1.0 - rb2));
        }
}

// Orbital m of a backflow determinant at x: value, gradient, Hessian
// [a*2 + b] and the Hessian's derivative along u, hu[a*2 + b] =
// Σ_c ∂_a∂_b∂_c φ u_c (OrbitalSet::evaluate_third_derivatives contracted
// with u).  Plane waves: ∂_a∂_b∂_c φ = -k_a k_b k_c φ' (φ' = -sin or cos);
// Gaussians e^{-α d²}: [4α²(δ_ac d_b + δ_bc d_a + δ_ab d_c) - 8α³ d_a d_b d_c] φ.
__device__ void bf_orbital3(const DevSys& s, const DevBF& D, int m, const double* x, const double* u, double* g,
                            double* h, double* hu) {
    if (D.type == 0) {
        const double kx = D.k[m * 2], ky = D.k[m * 2 + 1];
        double sn, c;
        sincos(kx * x[0] + ky * x[1], &sn, &c);
        const bool is_s = D.is_sin[m] != 0.0;
        const double v = is_s ? sn : c, dv = is_s ? c : -sn;
        const double k2[2] = {kx, ky};
        const double ku = kx * u[0] + ky * u[1];
        g[0] = kx * dv;
        g[1] = ky * dv;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                h[a * 2 + b] = -k2[a] * k2[b] * v;
                hu[a * 2 + b] = -k2[a] * k2[b] * dv * ku;
            }
    } else {
        const double al = D.alphas[m];
        double del[3] = {x[0] - D.centers[m * 2], x[1] - D.centers[m * 2 + 1], 0.0};
        min_image(s, del);
        const double phi = exp(-al * (del[0] * del[0] + del[1] * del[1]));
        const double du = del[0] * u[0] + del[1] * u[1];
        g[0] = -2.0 * al * del[0] * phi;
        g[1] = -2.0 * al * del[1] * phi;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                const double dab = a == b ? 1.0 : 0.0;
                h[a * 2 + b] = (4.0 * al * al * del[a] * del[b] - 2.0 * al * dab) * phi;
                hu[a * 2 + b] = (4.0 * al * al * (u[a] * del[b] + u[b] * del[a] + dab * du) -
                                 8.0 * al * al * al * del[a] * del[b] * du) *
                                phi;
            }
    }
}

// ∂(∇ ln|D|)/∂p and ∂(∇² ln|D|)/∂p of a backflow determinant for every
// optimisable channel parameter p of it, one CTA per walker, each parameter
// in turn (BackflowSlaterDeterminant::compute_parameter_gradient_derivatives
// and tangent_derivatives, backflow_slater_determinant.cpp:754-958).  The
// parameter moves the quasi-coordinates by ẋ_t = Σ_j ∂η(r_tj)/∂p r_tj, so
// with M[r][m] = φ_m(x_r) and A = M⁻¹ (committed):
//   Ṁ[r][m] = ∇φ_m(x_r)·ẋ_r,  Ȧ = -A Ṁ A,
//   Ḟ_iα = Σ_m Ȧ_mi ∂_αφ_m(x_i) + A_mi ∇∂_αφ_m(x_i)·ẋ_i,  Ṫ_i and Ġ^α alike,
// and for every affected particle k and direction β, with v, v̇ the Jacobian
// column of (k, β) and its parameter derivative (the pair tensors of ∂η/∂p,
// no identity part):
//   ∂_p ∂_kβ ln|D| = Σ_t Ḟ_t·v_t + F_t·v̇_t,
//   ∂_p ∂²_kβ ln|D| = Σ_t (Ḟ_t·S_t + F_t·Ṡ_t + 2 v̇_tᵀ T_t v_t + v_tᵀ Ṫ_t v_t)
//                    - 2 Σ_jr U̇_jr U_rj,   U_jr = Σ_α v_rα G^α_jr.
// Shared memory (doubles): 2 np + 20 N² + 22 N.  Outputs [q][p*2 + d][nw]
// for the backflow parameters q; other particles are left as they are.
template <int NT>
__global__ void __launch_bounds__(NT) bf_curvature_kernel(DevSys s, const double* records, int nw,
                                                          const DevOpt* opts, int nopt, double* dgrad,
                                                          double* dlap) {
    extern __shared__ __align__(16) double sm[];
    __shared__ double red[(NT / 32) * 4 + 4];
    const int w = blockIdx.x;
    if (w >= nw) return;
    const int np = s.np;
    const double* rec = records + static_cast<long>(w) * s.rec;
    double* pos = sm;
    for (int i = threadIdx.x; i < np * 2; i += NT) pos[i] = rec[s.o_pos + i];
    const long plane = static_cast<long>(np) * 2 * nw;
    for (int q = 0; q < nopt; ++q) {
        const DevOpt& o = opts[q];
        if (o.kind != 2) continue;
        const DevBF& D = s.bf[o.term];
        const DevBFCh& Cq = D.ch[o.ch];
        const int N = D.n, NN = N * N;
        double* x = pos + 2 * np;
        double* xd = x + 2 * N;
        double* A = xd + 2 * N;
        double* Ad = A + NN;
        double* Pm = Ad + NN;
        double* Gr = Pm + NN;     // ∇φ_m(x_r)       [(r*N + m)*2 + α]
        double* Hs = Gr + 2 * NN; // ∇∇φ_m(x_r)      [(r*N + m)*4 + αγ]
        double* Md = Hs + 4 * NN; // Ṁ[r][m]
        double* gd = Md + NN;     // (∇φ_m)˙(x_r)    [(r*N + m)*2 + α]
        double* hd = gd + 2 * NN; // (∇∇φ_m)˙(x_r)   [(r*N + m)*4 + αγ]
        double* G = hd + 4 * NN;  // G^α[j][r]       [α*NN + j*N + r]
        double* Gd = G + 2 * NN;
        double* T = Gd + 2 * NN;  // T_i [i*4 + αγ]
        double* Td = T + 4 * N;
        double* Fd = Td + 4 * N;  // Ḟ_i [i*2 + α]
        double* V = Fd + 2 * N;   // Jacobian column [β*2N + t*2 + α]
        double* Vd = V + 4 * N;
        const double* F = rec + D.oF;
        __syncthreads();
        for (int t = threadIdx.x; t < N; t += NT) {
            const int P = D.first + t;
            bf_row_x(s, D, pos, -1, nullptr, P, x + t * 2);
            double u0 = 0.0, u1 = 0.0;
            for (int j = Cq.sf; j < Cq.sl; ++j) {
                if (j == P) continue;
                double del[3] = {pos[P * 2] - pos[j * 2], pos[P * 2 + 1] - pos[j * 2 + 1], 0.0};
                min_image(s, del);
                const double r = sqrt(del[0] * del[0] + del[1] * del[1]);
                if (r >= Cq.L) continue;
                double de, d1, d2;
                bf_eta_dparam3(Cq, o.index, o.zs, r, de, d1, d2);
                u0 += de * del[0];
                u1 += de * del[1];
            }
            xd[t * 2] = u0;
            xd[t * 2 + 1] = u1;
        }
        for (int i = threadIdx.x; i < NN; i += NT) A[i] = rec[D.oA + i];
        __syncthreads();
        for (int e = threadIdx.x; e < NN; e += NT) {
            const int r = e / N, m = e % N;
            double g[2], h[4], hu[4];
            const double* u = xd + r * 2;
            bf_orbital3(s, D, m, x + r * 2, u, g, h, hu);
            Gr[e * 2] = g[0];
            Gr[e * 2 + 1] = g[1];
            Md[e] = g[0] * u[0] + g[1] * u[1];
            for (int a = 0; a < 2; ++a) {
                gd[e * 2 + a] = h[a * 2] * u[0] + h[a * 2 + 1] * u[1];
                for (int b = 0; b < 2; ++b) {
                    Hs[e * 4 + a * 2 + b] = h[a * 2 + b];
                    hd[e * 4 + a * 2 + b] = hu[a * 2 + b];
                }
            }
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NN; e += NT) {   // Pm = A Ṁ
            const int m = e / N, mp = e % N;
            double acc = 0.0;
            for (int r = 0; r < N; ++r) acc += A[m * N + r] * Md[r * N + mp];
            Pm[e] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < NN; e += NT) {   // Ȧ = -Pm A
            const int m = e / N, r = e % N;
            double acc = 0.0;
            for (int mp = 0; mp < N; ++mp) acc += Pm[m * N + mp] * A[mp * N + r];
            Ad[e] = -acc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < N; i += NT) {
            double f[2] = {0, 0}, tt[4] = {0, 0, 0, 0}, td[4] = {0, 0, 0, 0};
            for (int m = 0; m < N; ++m) {
                const double a = A[m * N + i], ad = Ad[m * N + i];
                const int e = i * N + m;
                for (int al = 0; al < 2; ++al) f[al] += ad * Gr[e * 2 + al] + a * gd[e * 2 + al];
                for (int ag = 0; ag < 4; ++ag) {
                    tt[ag] += a * Hs[e * 4 + ag];
                    td[ag] += ad * Hs[e * 4 + ag] + a * hd[e * 4 + ag];
                }
            }
            Fd[i * 2] = f[0];
            Fd[i * 2 + 1] = f[1];
            for (int ag = 0; ag < 4; ++ag) {
                T[i * 4 + ag] = tt[ag];
                Td[i * 4 + ag] = td[ag];
            }
        }
        for (int e = threadIdx.x; e < NN; e += NT) {
            const int j = e / N, r = e % N;
            double g0 = 0.0, g1 = 0.0, h0 = 0.0, h1 = 0.0;
            for (int m = 0; m < N; ++m) {
                const double a = A[m * N + j], ad = Ad[m * N + j];
                const int f = r * N + m;
                g0 += a * Gr[f * 2];
                g1 += a * Gr[f * 2 + 1];
                h0 += ad * Gr[f * 2] + a * gd[f * 2];
                h1 += ad * Gr[f * 2 + 1] + a * gd[f * 2 + 1];
            }
            G[e] = g0;
            G[NN + e] = g1;
            Gd[e] = h0;
            Gd[NN + e] = h1;
        }
        __syncthreads();
        for (int k = 0; k < np; ++k) {
            if (!bf_affects(D, k)) continue;
            const int tk = (k >= D.first && k < D.last) ? k - D.first : -1;
            // acc: 0-1 ∂_p of the gradient (β = 0, 1), 2-3 of the Laplacian
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            for (int t = threadIdx.x; t < N; t += NT) {
                double vt[2][2] = {{0, 0}, {0, 0}}, vd[2][2] = {{0, 0}, {0, 0}};
                const int P = D.first + t;
                const double* Ft = F + t * 2;
                const double* Fdt = Fd + t * 2;
                for (int c = 0; c < D.nch; ++c) {
                    const DevBFCh& Ch = D.ch[c];
                    const bool own = t == tk;
                    if (!own && (k < Ch.sf || k >= Ch.sl)) continue;
                    for (int j = own ? Ch.sf : k; j < (own ? Ch.sl : k + 1); ++j) {
                        if (own && j == k) continue;
                        const double* ri = own ? pos + k * 2 : pos + P * 2;
                        const double* rj = own ? pos + j * 2 : pos + k * 2;
                        double unused[2] = {0, 0}, B[4], S[4];
                        if (!bf_pair(s, Ch, ri, rj, 1.0, unused, B, S)) continue;
                        const double sg = own ? 1.0 : -1.0;
                        for (int be = 0; be < 2; ++be)
                            for (int a = 0; a < 2; ++a) {
                                vt[be][a] += sg * B[a * 2 + be];
                                acc[2 + be] += Fdt[a] * S[a * 2 + be];
                            }
                        if (c != o.ch) continue;
                        double del[3] = {ri[0] - rj[0], ri[1] - rj[1], 0.0};
                        min_image(s, del);
                        const double r = sqrt(del[0] * del[0] + del[1] * del[1]);
                        double de, d1, d2, Bd[4], Sd[4];
                        bf_eta_dparam3(Ch, o.index, o.zs, r, de, d1, d2);
                        bf_tensors(de, d1, d2, del, r, Bd, Sd);
                        for (int be = 0; be < 2; ++be)
                            for (int a = 0; a < 2; ++a) {
                                vd[be][a] += sg * Bd[a * 2 + be];
                                acc[2 + be] += Ft[a] * Sd[a * 2 + be];
                            }
                    }
                }
                if (t == tk) {
                    vt[0][0] += 1.0;
                    vt[1][1] += 1.0;
                }
                for (int be = 0; be < 2; ++be) {
                    V[be * 2 * N + t * 2] = vt[be][0];
                    V[be * 2 * N + t * 2 + 1] = vt[be][1];
                    Vd[be * 2 * N + t * 2] = vd[be][0];
                    Vd[be * 2 * N + t * 2 + 1] = vd[be][1];
                    acc[be] += Fdt[0] * vt[be][0] + Fdt[1] * vt[be][1] + Ft[0] * vd[be][0] + Ft[1] * vd[be][1];
                    const double* Tt = T + t * 4;
                    const double* Tdt = Td + t * 4;
                    for (int a = 0; a < 2; ++a)
                        for (int g = 0; g < 2; ++g)
                            acc[2 + be] += 2.0 * vd[be][a] * Tt[a * 2 + g] * vt[be][g] +
                                           vt[be][a] * Tdt[a * 2 + g] * vt[be][g];
                }
            }
            __syncthreads();
            for (int e = threadIdx.x; e < NN; e += NT) {
                const int j = e / N, r = e % N;
                for (int be = 0; be < 2; ++be) {
                    const double* Vb = V + be * 2 * N;
                    const double* Vdb = Vd + be * 2 * N;
                    const double urj = Vb[j * 2] * G[r * N + j] + Vb[j * 2 + 1] * G[NN + r * N + j];
                    const double udjr = Vdb[r * 2] * G[e] + Vdb[r * 2 + 1] * G[NN + e] + Vb[r * 2] * Gd[e] +
                                        Vb[r * 2 + 1] * Gd[NN + e];
                    acc[2 + be] -= 2.0 * udjr * urj;
                }
            }
            block_sum<NT>(acc, red);
            if (threadIdx.x == 0) {
                const long base = q * plane + static_cast<long>(k) * 2 * nw + w;
                dgrad[base] = acc[0];
                dgrad[base + nw] = acc[1];
                dlap[base] = acc[2];
                dlap[base + nw] = acc[3];
            }
            __syncthreads();
        }
    }
}

// pair sum of du/dp over the term's pairs (minus, for an image sum, the
// breakup's long-range part and limit inside r_cut, zero outside) plus the
// image sum's k-space part, sum_k w'_k |rho_a|^2 or 2 Re rho_a rho_b*
// (kspace_pair_sum.cpp:109-122, :303-313).
template <int NT>
__global__ void __launch_bounds__(NT) param_kernel(DevSys s, const double* records, int nw, const DevOpt* opts,
                                                   int nopt, double* out) {
    __shared__ double pos[2 * 256];
    __shared__ double red[NT];
    const int w = blockIdx.x;
    if (w >= nw || s.np > 256) return;
    const double* rec = records + static_cast<long>(w) * s.rec;
    for (int i = threadIdx.x; i < s.np * 2; i += NT) pos[i] = rec[s.o_pos + i];
    __syncthreads();
    for (int q = 0; q < nopt; ++q) {
        const DevOpt& o = opts[q];
        if (o.kind == 1) continue;   // orbital widths: orbital_param_kernel
        double acc = 0.0;
        if (o.kind == 2) {
            // Σ_P Σ_j (F_P · r_Pj) ∂η(r_Pj)/∂p over the channel's sources j ≠ P
            // (BackflowTransformation::parameter_derivatives,
            // backflow_transformation.cpp:284-312; F_P the committed row of F)
            const DevBF& D = s.bf[o.term];
            const DevBFCh& C = D.ch[o.ch];
            const double* F = rec + D.oF;
            const int ns = C.sl - C.sf;
            for (int e = threadIdx.x; e < D.n * ns; e += NT) {
                const int t = e / ns, j = C.sf + e % ns, P = D.first + t;
                if (j == P) continue;
                double del[3];
                const double r = fold_dist(s, pos + P * 2, pos + j * 2, del);
                if (r >= C.L) continue;
                acc += (F[t * 2] * del[0] + F[t * 2 + 1] * del[1]) * bf_eta_dparam(C, o.index, o.zs, r);
            }
        }
        const DevTerm& T = s.terms[o.kind == 0 ? o.term : 0];
        for (int pp = 0; o.kind == 0 && pp < T.npairs; ++pp) {
            const int af = T.pairs[pp][0], al = T.pairs[pp][1], bf = T.pairs[pp][2], bl = T.pairs[pp][3];
            const bool same = af == bf && al == bl;
            const int na = al - af, nb = bl - bf;
            const int tot = na * nb;
            for (int e = threadIdx.x; e < tot; e += NT) {
                const int i = af + e / nb, j = bf + e % nb;
                if (same && j <= i) continue;
                double del[3];
                const double r = fold_dist(s, pos + i * 2, pos + j * 2, del);
                double v = dudp(T, o, r);
                if (T.image) v = r < o.sp.r_cut ? v - (o.inf + spline1(o.sp, r)) : 0.0;
                acc += v;
            }
        }
        if (o.kind == 0 && T.image) {
            const int ga = s.group_of[T.pairs[0][0]], gb = s.group_of[T.pairs[0][2]];
            const double* ra = rec + s.o_rho + 2 * ga * s.nkJ;
            const double* rb = rec + s.o_rho + 2 * gb * s.nkJ;
            for (int k = threadIdx.x; k < s.nkJ; k += NT) {
                if (T.same0) acc += o.kw[k] * (ra[k] * ra[k] + ra[s.nkJ + k] * ra[s.nkJ + k]);
                else acc += 2.0 * o.kw[k] * (ra[k] * rb[k] + ra[s.nkJ + k] * rb[s.nkJ + k]);
            }
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int h = NT / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[static_cast<long>(q) * nw + w] = red[0];
        __syncthreads();
    }
}

// The shared width alpha of a Gaussian orbital block (kind-1 parameters), for
// the walkers blockIdx.x, blockIdx.x + gridDim.x, ...; scratch holds three
// N x N matrices per CTA.  With D_{c,a} = phi_a(r_c), phi = exp(-alpha |Δ|^2)
// at the minimum image Δ = r_c - R_a, and A = D^-1 (A[m N + c]):
//   O       = sum_{c,a} A_{a,c} dD_{c,a},  dD = d phi / d alpha = -|Δ|^2 phi
//   dA      = -A dD A
//   dG_d(j) = sum_m dA_{m,j} d_d phi_m(r_j) + A_{m,j} d_alpha d_d phi_m(r_j)
//   dL_d(j) = sum_m dA_{m,j} d2_d phi_m(r_j) + A_{m,j} d_alpha d2_d phi_m(r_j) - 2 G_d(j) dG_d(j)
// (slater_determinant.cpp:98-157, :159-250; orbital_set.h:250-286).
template <int NT>
__global__ void __launch_bounds__(NT) orbital_param_kernel(DevSys s, const double* records, int nw,
                                                           const DevOpt* opts, int nopt, double* out,
                                                           double* dgrad, double* dlap, double* scratch) {
    __shared__ double red[NT];
    const long n2 = static_cast<long>(s.maxN) * s.maxN;
    double* dD = scratch + blockIdx.x * 3 * n2;
    double* Y = dD + n2;
    double* dA = Y + n2;
    const long plane = static_cast<long>(s.np) * 2 * nw;
    for (int w = blockIdx.x; w < nw; w += gridDim.x) {
        const double* rec = records + static_cast<long>(w) * s.rec;
        const double* pos = rec + s.o_pos;
        for (int q = 0; q < nopt; ++q) {
            const DevOpt& o = opts[q];
            if (o.kind != 1) continue;
            const DevBlock& B = s.blocks[o.term];
            const int N = B.n;
            const double* A = rec + B.oA;
            const double al = B.alphas[0];
            double acc = 0.0;
            for (int e = threadIdx.x; e < N * N; e += NT) {
                const int c = e / N, a = e % N;
                double del[3] = {pos[(B.first + c) * 2] - B.centers[a * 2],
                                 pos[(B.first + c) * 2 + 1] - B.centers[a * 2 + 1], 0.0};
                min_image(s, del);
                const double r2 = del[0] * del[0] + del[1] * del[1];
                dD[e] = -r2 * exp(-al * r2);
                acc += A[a * N + c] * dD[e];
            }
            red[threadIdx.x] = acc;
            __syncthreads();
            for (int h = NT / 2; h > 0; h >>= 1) {
                if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
                __syncthreads();
            }
            if (threadIdx.x == 0 && out) out[static_cast<long>(q) * nw + w] = red[0];
            __syncthreads();
            if (!dgrad && !dlap) continue;
            for (int e = threadIdx.x; e < N * N; e += NT) {   // Y = dD A
                const int c = e / N, j = e % N;
                double t = 0.0;
                for (int a = 0; a < N; ++a) t = fma(dD[c * N + a], A[a * N + j], t);
                Y[e] = t;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < N * N; e += NT) {   // dA = -A Y
                const int m = e / N, j = e % N;
                double t = 0.0;
                for (int c = 0; c < N; ++c) t = fma(A[m * N + c], Y[c * N + j], t);
                dA[e] = -t;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < N * 2; e += NT) {
                const int j = e / 2, d = e % 2;
                const int particle = B.first + j;
                const double xj = pos[particle * 2], yj = pos[particle * 2 + 1];
                double dG = 0.0, dL = 0.0;
                for (int m = 0; m < N; ++m) {
                    double del[3] = {xj - B.centers[m * 2], yj - B.centers[m * 2 + 1], 0.0};
                    min_image(s, del);
                    const double r2 = del[0] * del[0] + del[1] * del[1];
                    const double phi = exp(-al * r2), dd = del[d];
                    const double g = -2.0 * al * dd * phi;
                    const double l = (4.0 * al * al * dd * dd - 2.0 * al) * phi;
                    const double dg = -2.0 * dd * phi * (1.0 - al * r2);
                    const double dl = phi * (8.0 * al * dd * dd - 2.0 - r2 * (4.0 * al * al * dd * dd - 2.0 * al));
                    const double a = A[m * N + j], da = dA[m * N + j];
                    dG += da * g + a * dg;
                    dL += da * l + a * dl;
                }
                const long idx = q * plane + (static_cast<long>(particle) * 2 + d) * nw + w;
                if (dgrad) dgrad[idx] = dG;
                if (dlap) dlap[idx] = dL - 2.0 * rec[s.o_sg + particle * 2 + d] * dG;
            }
            __syncthreads();
        }
    }
}

// FP64 CUDA-core peak probe: every thread runs 8 independent FMA chains of
// `iters` steps (no memory traffic); out gets a sum so the work is kept.
__global__ void __launch_bounds__(256) fp64_fma_kernel(int iters, double* out) {
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = 1.0 + 1e-9 * (threadIdx.x + k);
    const double m = 0.999999999, c = 1e-12;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], m, c);
    }
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) t += a[k];
    if (t == 12345.678) out[0] = t;   // never true; keeps the chains live
}

// Potential energy of stored configurations (Hamiltonian::evaluate_potential,
// src/hamiltonian/hamiltonian_component.h:165-403): configuration c is
// rows[idx[c]] (positions [np][2]); the local energy's potential terms with
// zero derivative planes, so the kinetic part adds nothing.
template <int NT>
__global__ void __launch_bounds__(NT) potential_kernel(DevSys s, const double* rows, const int* idx, int n,
                                                       const int2* pairs, int npair, double* out) {
    extern __shared__ __align__(16) double sm[];
    const int c = blockIdx.x;
    if (c >= n) return;
    const Smem v = view(s, sm);
    const double* r = rows + static_cast<long>(idx[c]) * s.np * 2;
    for (int i = threadIdx.x; i < s.np * 2; i += NT) {
        v.pos[i] = r[i];
        v.jg[i] = v.jl[i] = v.kg[i] = v.kl[i] = v.sg[i] = v.sl[i] = 0.0;
        if (s.cplx) v.pg[i] = v.pl[i] = 0.0;
    }
    __syncthreads();
    const double e = local_energy<NT>(s, v, pairs, npair);
    if (threadIdx.x == 0) out[c] = e;
}

template <int NT>
__global__ void __launch_bounds__(NT) measure_kernel(DevSys s, double* records, int nw,
                                                     const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_hot<NT>(s, rec, sm);
    const Smem v = view(s, sm);
    refresh_all<NT>(s, v, rec);
    const double el = local_energy<NT>(s, v, pairs, npair);
    if (threadIdx.x == 0) v.scal[S_EL] = el;
    store_hot<NT>(s, rec, sm);
}

template <int NT>
__global__ void __launch_bounds__(NT) move_kernel(DevSys s, double* records, int nw, int p,
                                                  const double* new_pos, const uint8_t* accept,
                                                  double* out) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_hot<NT>(s, rec, sm);
    const Smem v = view(s, sm);
    if (threadIdx.x == 0) {
        v.newpos[0] = new_pos[w];
        v.newpos[1] = new_pos[nw + w];
        v.misc[M_ERR] = 0.0;
    }
    __syncthreads();
    ratio_step<NT>(s, v, p, false);
    if (threadIdx.x == 0) {
        // log ratio, phase, new ∇ln ψ (dim), new ∂² ln ψ (dim), per walker
        out[0 * nw + w] = v.misc[M_LOGR];
        out[1 * nw + w] = v.misc[M_PHASE];
        out[2 * nw + w] = v.misc[M_SGX] + v.misc[M_JGX] + v.misc[M_KGX];
        out[3 * nw + w] = v.misc[M_SGY] + v.misc[M_JGY] + v.misc[M_KGY];
        out[4 * nw + w] = v.misc[M_SLX] + v.misc[M_JLX] + v.misc[M_KLX];
        out[5 * nw + w] = v.misc[M_SLY] + v.misc[M_JLY] + v.misc[M_KLY];
    }
    if (accept != nullptr && accept[w] != 0) commit_step<NT>(s, v, rec, p);
    store_hot<NT>(s, rec, sm);
}

// Fused sweep kernel.  mode 0: VMC step (n_sub sweeps, then refresh + E_L);
// mode 1: DMC advance (per sweep: refresh + E_L + branch factor).
template <int NT>
__device__ __forceinline__ void sweep_walker(const DevSys& s, double* records, int w, const double* randoms,
                                             long stride, const SweepParams& prm, const int2* pairs, int npair,
                                             double* sm) {
    double* rec = records + static_cast<long>(w) * s.rec;
    load_hot<NT>(s, rec, sm);
    const Smem v = view(s, sm);
    const int np = s.np;
    const bool dmc = prm.mode == 1;
    const bool drift = dmc || prm.drift != 0;
    if (threadIdx.x == 0) {
        v.scal[S_NACC] = 0.0;
        v.scal[S_NCUT] = 0.0;
        if (dmc) {
            v.scal[S_RRP] = 0.0;
            v.scal[S_RRA] = 0.0;
            v.scal[S_WEIGHT] = 1.0;
            v.scal[S_EPREV] = v.scal[S_EL];
        }
        v.misc[M_ERR] = 0.0;
    }
    __syncthreads();
    for (int sub = 0; sub < prm.n_sub; ++sub) {
        const double* rnd = randoms + static_cast<long>(sub) * np * 3 * stride;
        for (int p = 0; p < np; ++p) {
            if (drift) refresh_particle<NT>(s, v, rec, p);
            if (threadIdx.x == 0) {
                const double* g = rnd + static_cast<long>(p) * 3 * stride;
                const double tm = prm.tau * s.inv_mass[p * 2];
                const double gx = v.sg[p * 2] + v.jg[p * 2] + v.kg[p * 2];
                const double gy = v.sg[p * 2 + 1] + v.jg[p * 2 + 1] + v.kg[p * 2 + 1];
                double sc = tm;
                if (dmc) {
                    const double vsq = gx * gx + gy * gy;
                    sc = vsq < 1e-10 ? tm : (-1.0 + sqrt(1.0 + 2.0 * tm * vsq)) / vsq;
                }
                v.misc[M_SCFWD] = sc;
                const double sig0 = prm.sigma[p * 2], sig1 = prm.sigma[p * 2 + 1];
                if (drift) {
                    const double t0 = dmc ? sc : prm.tau * s.inv_mass[p * 2];
                    const double t1 = dmc ? sc : prm.tau * s.inv_mass[p * 2 + 1];
                    v.newpos[0] = fma(sig0, g[0 * stride + w], fma(t0, gx, v.pos[p * 2]));
                    v.newpos[1] = fma(sig1, g[1 * stride + w], fma(t1, gy, v.pos[p * 2 + 1]));
                } else {
                    v.newpos[0] = fma(sig0, g[0 * stride + w], v.pos[p * 2]);
                    v.newpos[1] = fma(sig1, g[1 * stride + w], v.pos[p * 2 + 1]);
                }
                v.misc[M_U] = g[2 * stride + w];
                v.misc[M_GOX] = gx;   // current total gradient, for the Green's function
                v.misc[M_GOY] = gy;
            }
            __syncthreads();
            ratio_step<NT>(s, v, p, drift);
            if (threadIdx.x == 0) {
                const double logr = v.misc[M_LOGR];
                const double u = v.misc[M_U];
                const double gx = v.misc[M_GOX], gy = v.misc[M_GOY];
                const double ngx = v.misc[M_SGX] + v.misc[M_JGX] + v.misc[M_KGX];
                const double ngy = v.misc[M_SGY] + v.misc[M_JGY] + v.misc[M_KGY];
                const double dx = v.newpos[0] - v.pos[p * 2], dy = v.newpos[1] - v.pos[p * 2 + 1];
                const double tm0 = prm.tau * s.inv_mass[p * 2], tm1 = prm.tau * s.inv_mass[p * 2 + 1];
                bool acc;
                if (dmc) {
                    acc = false;
                    // a real ratio's phase is 0 or π: the fixed-node gate (cos φ < ε)
                    // fixed phase (complex ψ) has no gate
                    if (s.cplx || v.misc[M_PHASE] == 0.0) {
                        const double vsq = ngx * ngx + ngy * ngy;
                        const double sb = vsq < 1e-10 ? tm0 : (-1.0 + sqrt(1.0 + 2.0 * tm0 * vsq)) / vsq;
                        const double sf = v.misc[M_SCFWD];
                        double lc = 0.0;
                        if (tm0 > 0.0) {
                            const double df = sf * gx, db = sb * ngx;
                            lc += (-dx * (df + db) + 0.5 * (df * df - db * db)) / tm0;
                        }
                        if (tm1 > 0.0) {
                            const double df = sf * gy, db = sb * ngy;
                            lc += (-dy * (df + db) + 0.5 * (df * df - db * db)) / tm1;
                        }
                        const double la = 2.0 * logr + lc;
                        acc = la >= 0.0 || u < exp(la);
                    }
                    const double rr = tm0 * dx * dx + tm1 * dy * dy;
                    v.scal[S_RRP] += rr;
                    if (acc) v.scal[S_RRA] += rr;
                } else if (prm.drift) {
                    double lc = -dx * (gx + ngx) + 0.5 * tm0 * (gx * gx - ngx * ngx);
                    lc += -dy * (gy + ngy) + 0.5 * tm1 * (gy * gy - ngy * ngy);
                    const double la = 2.0 * logr + lc;
                    acc = la >= 0.0 || u < exp(la);
                } else {
                    acc = u < exp(2.0 * logr);
                }
                v.misc[M_ACCEPT] = acc ? 1.0 : 0.0;
                if (acc) v.scal[S_NACC] += 1.0;
            }
            __syncthreads();
            if (v.misc[M_ACCEPT] != 0.0) commit_step<NT>(s, v, rec, p);
        }
        if (dmc || sub == prm.n_sub - 1) {
            refresh_all<NT>(s, v, rec);
            const double el = local_energy<NT>(s, v, pairs, npair);
            if (threadIdx.x == 0) {
                v.scal[S_EL] = el;
                if (dmc) {
                    const double enew = el, eold = v.scal[S_EPREV];
                    double half_tau = 0.5 * prm.tau;
                    const double x = fmax(prm.eref - enew, prm.eref - eold);
                    if (x > prm.e_max)
                        half_tau = 0.0;
                    else if (x > prm.e_cut)
                        half_tau *= 1.0 - (x - prm.e_cut) / (prm.e_max - prm.e_cut);
                    v.scal[S_WEIGHT] *= exp(half_tau * (2.0 * prm.etrial - enew - eold));
                    if (x > prm.e_cut) v.scal[S_NCUT] += 1.0;
                    v.scal[S_EPREV] = enew;
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        if (dmc && prm.tau > 0.0) v.scal[S_AGE] = v.scal[S_RRP] > 0.0 ? 0.0 : v.scal[S_AGE] + 1.0;
        if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
    }
    store_hot<NT>(s, rec, sm);
}

// One CTA of NT threads per walker.
template <int NT>
__global__ void __launch_bounds__(NT) sweep_kernel(DevSys s, double* records, int nw,
                                                   const double* randoms, long stride,
                                                   SweepParams prm, const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    sweep_walker<NT>(s, records, w, randoms, stride, prm, pairs, npair, sm);
}

// Packed generic sweeps of several contexts, 32 threads per walker
// (BatchJob, alea_kernels.h).
template <int NT>
__global__ void __launch_bounds__(NT) sweep_batch_kernel(const BatchJob* __restrict__ jobs, int n_jobs, int total,
                                                         int* next) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int slot;
    for (bool first = true;; first = false) {
        const int w = batch_next(total, next, &slot, first);
        if (w < 0) return;
        const BatchJob& J = jobs[batch_job_of(jobs, n_jobs, w)];
        sweep_walker<NT>(*J.sys, J.records, w - J.first, J.randoms, J.stride, J.prm, J.pairs, J.npair, sm);
    }
}

// ───────────────────────── launchers ────────────────────────────────────

#define ALEA_LAUNCH(nt, KERNEL, grid, smem, st, ...)                                     \
    do {                                                                                 \
        if ((nt) == 32) KERNEL<32><<<(grid), 32, (smem), (st)>>>(__VA_ARGS__);           \
        else if ((nt) == 64) KERNEL<64><<<(grid), 64, (smem), (st)>>>(__VA_ARGS__);      \
        else KERNEL<128><<<(grid), 128, (smem), (st)>>>(__VA_ARGS__);                    \
    } while (0)

// The dynamic shared-memory cap is a property of each kernel function, shared
// by every context on the device: it only ever grows, under a lock, so that
// contexts of different systems created on different threads (a server's
// workers) never lower it beneath a launch in flight.
cudaError_t reserve_smem(size_t smem) {
    static std::mutex mu;
    static size_t reserved[64] = {};   // per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (smem <= reserved[dev]) return cudaSuccess;
    const int b = static_cast<int>(smem);
    const void* kernels[] = {
        reinterpret_cast<const void*>(evaluate_kernel<32>), reinterpret_cast<const void*>(measure_kernel<32>),
        reinterpret_cast<const void*>(move_kernel<32>), reinterpret_cast<const void*>(sweep_kernel<32>),
        reinterpret_cast<const void*>(evaluate_kernel<64>), reinterpret_cast<const void*>(measure_kernel<64>),
        reinterpret_cast<const void*>(move_kernel<64>), reinterpret_cast<const void*>(sweep_kernel<64>),
        reinterpret_cast<const void*>(evaluate_kernel<128>), reinterpret_cast<const void*>(measure_kernel<128>),
        reinterpret_cast<const void*>(move_kernel<128>), reinterpret_cast<const void*>(sweep_kernel<128>),
        reinterpret_cast<const void*>(potential_kernel<32>), reinterpret_cast<const void*>(potential_kernel<64>),
        reinterpret_cast<const void*>(potential_kernel<128>), reinterpret_cast<const void*>(sweep_batch_kernel<32>),
        reinterpret_cast<const void*>(sweep_batch_kernel<64>), reinterpret_cast<const void*>(sweep_batch_kernel<128>)};
    for (const void* k : kernels) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = reserve_smem_fast(smem);
    if (e == cudaSuccess) e = reserve_smem_boson(smem);
    if (e == cudaSuccess) e = reserve_smem_f32(smem);
    if (e == cudaSuccess) reserved[dev] = smem;
    return e;
}

cudaError_t launch_param_derivatives(int nw, cudaStream_t st, const DevSys& s, const double* records,
                                     const DevOpt* opts, int nopt, double* out) {
    if (nw < 1 || nopt < 1) return cudaSuccess;
    param_kernel<128><<<nw, 128, 0, st>>>(s, records, nw, opts, nopt, out);
    return cudaGetLastError();
}

cudaError_t launch_orbital_param_derivatives(int nw, int grid, cudaStream_t st, const DevSys& s,
                                            const double* records, const DevOpt* opts, int nopt, double* out,
                                            double* dgrad, double* dlap, double* scratch) {
    if (nw < 1 || nopt < 1) return cudaSuccess;
    orbital_param_kernel<128><<<grid, 128, 0, st>>>(s, records, nw, opts, nopt, out, dgrad, dlap, scratch);
    return cudaGetLastError();
}

cudaError_t launch_param_grad_derivatives(int nw, cudaStream_t st, const DevSys& s, const double* records,
                                          const DevOpt* opts, int nopt, double* dgrad, double* dlap) {
    if (nw < 1 || nopt < 1) return cudaSuccess;
    param_grad_kernel<64><<<nw, 64, 0, st>>>(s, records, nw, opts, nopt, dgrad, dlap);
    return cudaGetLastError();
}

size_t bf_curvature_smem(const DevSys& s) {
    int n = 0;
    for (int d = 0; d < s.nbf; ++d) n = std::max(n, s.bf[d].n);
    // positions 2 np; A, Ȧ, A Ṁ, Ṁ (N² each), ∇φ, ∇φ˙, G, Ġ (2N²), ∇∇φ, ∇∇φ˙ (4N²);
    // x, ẋ, Ḟ (2N), T, Ṫ, the two Jacobian columns and their derivatives (4N)
    return 8 * (2 * static_cast<size_t>(s.np) + 20 * static_cast<size_t>(n) * n + 22 * static_cast<size_t>(n));
}

cudaError_t launch_bf_curvature(int nw, cudaStream_t st, const DevSys& s, const double* records, const DevOpt* opts,
                                int nopt, double* dgrad, double* dlap) {
    if (nw < 1 || nopt < 1 || s.nbf < 1) return cudaSuccess;
    const size_t smem = bf_curvature_smem(s);
    {   // raised only, so a context on another thread never sees its reservation shrink
        static std::mutex mu;
        static size_t reserved[64] = {};
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
        std::lock_guard<std::mutex> lk(mu);
        if (smem > reserved[dev]) {
            const cudaError_t e = cudaFuncSetAttribute(bf_curvature_kernel<128>,
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(smem));
            if (e != cudaSuccess) return e;
            reserved[dev] = smem;
        }
    }
    bf_curvature_kernel<128><<<nw, 128, smem, st>>>(s, records, nw, opts, nopt, dgrad, dlap);
    return cudaGetLastError();
}

cudaError_t measure_fp64_peak(int device, double* tflops) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t st;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return e;
    double* out = nullptr;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    e = cudaMallocAsync(&out, sizeof(double), st);
    const int grid = sms * 8, iters = 1 << 14;
    double best = 0.0;
    for (int rep = 0; e == cudaSuccess && rep < 4; ++rep) {   // the first launch warms up
        cudaEventRecord(e0, st);
        fp64_fma_kernel<<<grid, 256, 0, st>>>(iters, out);
        cudaEventRecord(e1, st);
        e = cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8.0 * iters * grid * 256.0;
        if (rep > 0 && ms > 0.0f) best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    if (out) cudaFreeAsync(out, st);
    cudaStreamSynchronize(st);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(st);
    *tflops = best;
    return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t launch_potential(int nt, int n, size_t smem, cudaStream_t st, const DevSys& s, const double* rows,
                             const int* idx, const int2* pairs, int npair, double* out) {
    if (n < 1) return cudaSuccess;
    ALEA_LAUNCH(nt, potential_kernel, n, smem, st, s, rows, idx, n, pairs, npair, out);
    return cudaGetLastError();
}

cudaError_t launch_evaluate(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                            double* records, const int2* pairs, int npair) {
    ALEA_LAUNCH(nt, evaluate_kernel, nw, smem, st, s, records, nw, pairs, npair);
    return cudaGetLastError();
}

cudaError_t launch_measure(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                           double* records, const int2* pairs, int npair) {
    ALEA_LAUNCH(nt, measure_kernel, nw, smem, st, s, records, nw, pairs, npair);
    return cudaGetLastError();
}

cudaError_t launch_move(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                        double* records, int p, const double* new_pos, const uint8_t* accept,
                        double* out) {
    ALEA_LAUNCH(nt, move_kernel, nw, smem, st, s, records, nw, p, new_pos, accept, out);
    return cudaGetLastError();
}

cudaError_t launch_sweep(int nt, int nw, size_t smem, cudaStream_t st, const DevSys& s,
                         double* records, const double* randoms, long stride,
                         const SweepParams& prm, const int2* pairs, int npair) {
    if (s.f32)   // the FP32 form keeps no FP64 orbital rows: no other sweep may run on its records
        return launch_sweep_f32(nw, st, s, records, randoms, stride, prm, pairs, npair);
    const char* e = std::getenv("ALEA_GPU_SWEEP");
    const bool one_warp = e == nullptr || std::strcmp(e, "generic") != 0;
    if (one_warp && nt == 32 && fast_sweep_eligible(s))
        return launch_sweep_fast(nw, smem, st, s, records, randoms, stride, prm, pairs, npair);
    if (one_warp && boson_sweep_eligible(s))
        return launch_sweep_boson(nw, st, s, records, randoms, stride, prm, pairs, npair);
    ALEA_LAUNCH(nt, sweep_kernel, nw, smem, st, s, records, nw, randoms, stride, prm, pairs, npair);
    return cudaGetLastError();
}
cudaError_t launch_sweep_generic_batch(int nt, const BatchJob* jobs, int n_jobs, int total, int grid, size_t smem,
                                       int* next, cudaStream_t st) {
    ALEA_LAUNCH(nt, sweep_batch_kernel, grid, smem, st, jobs, n_jobs, total, next);
    return cudaGetLastError();
}

int batch_ctas_per_sm(int nt, size_t smem) {
    int n = 0;
    cudaError_t e = cudaSuccess;
    if (nt == 32) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_batch_kernel<32>, 32, smem);
    else if (nt == 64) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_batch_kernel<64>, 64, smem);
    else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_batch_kernel<128>, 128, smem);
    return e == cudaSuccess ? std::max(n, 1) : 1;
}

#undef ALEA_LAUNCH

// One sweep's (or several sweeps') random numbers per stream: stream t fills
// its crowd [w0, w1) of min(n_streams, nw) even splits in the reference's
// order (per particle: dim·n Gaussians dimension-major, then n uniforms).
// out[(sweep*np + p)*(dim+1)*stride + d*stride + w].
__global__ void draw_kernel(uint64_t* states, int n_streams, int nw, int np, long stride,
                            int n_sweeps, const uint64_t* zk, const double* zw, const double* zf,
                            double zr, double* out, int dim) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_active = n_streams < nw ? n_streams : nw;
    if (t >= n_active) return;
    const long base = nw / n_active, rem = nw % n_active;
    const long w0 = t * base + (t < rem ? t : rem);
    const long cnt = base + (t < rem ? 1 : 0);
    Xo r{states[t * 4 + 0], states[t * 4 + 1], states[t * 4 + 2], states[t * 4 + 3]};
    for (int sw = 0; sw < n_sweeps; ++sw)
        for (int p = 0; p < np; ++p) {
            double* row = out + (static_cast<long>(sw) * np + p) * (dim + 1) * stride;
            for (int d = 0; d < dim; ++d)
                for (long w = w0; w < w0 + cnt; ++w) row[d * stride + w] = xo_gaussian(r, zk, zw, zf, zr);
            for (long w = w0; w < w0 + cnt; ++w) row[dim * stride + w] = xo_uniform(r);
        }
    states[t * 4 + 0] = r.s0;
    states[t * 4 + 1] = r.s1;
    states[t * 4 + 2] = r.s2;
    states[t * 4 + 3] = r.s3;
}

// dst record j ← src record src_idx[j] (branching), 16-byte vector copies.
__global__ void gather_kernel(double* dst, const double* src, const int* src_idx, int n, long rec) {
    const int j = blockIdx.x;
    if (j >= n) return;
    const double2* a = reinterpret_cast<const double2*>(src + static_cast<long>(src_idx[j]) * rec);
    double2* b = reinterpret_cast<double2*>(dst + static_cast<long>(j) * rec);
    for (long i = threadIdx.x; i < rec / 2; i += blockDim.x) b[i] = a[i];
}

// Scalar slot of every walker into a packed [nw] array.
__global__ void scalar_kernel(const double* records, int nw, long rec, int offset, double* out) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nw) out[w] = records[static_cast<long>(w) * rec + offset];
}

// Walker-major record planes [w][i] ↔ SoA [i*nw + w] (positions, gradients).
__global__ void to_soa_kernel(const double* records, int nw, long rec, int offset, int n,
                              double* out) {
    const long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<long>(n) * nw) return;
    const int i = static_cast<int>(e / nw), w = static_cast<int>(e % nw);
    out[e] = records[static_cast<long>(w) * rec + offset + i];
}
__global__ void from_soa_kernel(double* records, int nw, long rec, int offset, int n,
                                const double* in) {
    const long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<long>(n) * nw) return;
    const int i = static_cast<int>(e / nw), w = static_cast<int>(e % nw);
    records[static_cast<long>(w) * rec + offset + i] = in[e];
}

__global__ void to_rows_kernel(const double* records, int nw, long rec, int offset, int n, double* out) {
    const long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<long>(n) * nw) return;
    const int w = static_cast<int>(e / n), i = static_cast<int>(e % n);
    out[e] = records[static_cast<long>(w) * rec + offset + i];
}
__global__ void from_rows_kernel(double* records, int nw, long rec, int offset, int n, const double* rows,
                                 int n_rows) {
    const long e = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= static_cast<long>(n) * nw) return;
    const int w = static_cast<int>(e / n), i = static_cast<int>(e % n);
    records[static_cast<long>(w) * rec + offset + i] = rows[static_cast<long>(w % n_rows) * n + i];
}
__global__ void cycle_index_kernel(int* idx, int nw, int n_src) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nw) idx[w] = w % n_src;
}

__global__ void set_scalar_kernel(double* records, int nw, long rec, int offset, double value) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w < nw) records[static_cast<long>(w) * rec + offset] = value;
}

}  // namespace alea_gpu
