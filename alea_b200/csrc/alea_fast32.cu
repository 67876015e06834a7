// The FP32 form of the one-warp sweep (sm_100a), for the plane-wave systems
// of the FP64 one-warp sweep (real plane-wave determinants, Padé/Drummond
// pair terms by group, at most 64 particles).  No reference counterpart: the reference is FP64
// throughout.
//
// In FP32: the inverses A (shared memory), orbital values and derivatives,
// the ratio, the rank-one Sherman-Morrison update, the pair-Jastrow radial
// functions and the image-sum terms of every move.  Angles are formed and
// reduced modulo 2π in FP64 before the single-precision sincos, and every
// sum over orbitals, partners or k-vectors is accumulated in FP64.
// In FP64: positions and proposals (so the random walk consumes the same
// randoms as the FP64 path), the pair-Jastrow gradient planes and ρ(k) (FP32
// changes added to FP64 totals), the full inverse recomputation every 64
// updates or on a trigger (orbital rows recomputed in FP64 from the
// positions, in-place Gauss-Jordan in FP64, rounded to FP32), log|det|, and
// the local energy with the DMC weight (orbital derivatives recomputed in
// FP64, ρ(k) recomputed from the positions, Ewald in FP64).  No orbital rows
// are kept in HBM: the FP64 rows would be stale, so the context re-evaluates
// before any FP64 path reads them (alea_gpu_set_precision).
//
// Steps and citations as in alea_fast.cu (src/qmc/vmc.cpp:82-155,
// src/qmc/dmc.cpp:203-337, src/wavefunction/slater_determinant.cpp:395-993,
// src/wavefunction/pade_jastrow.cpp:347-634, kspace_pair_sum.cpp:157-301).
#include "alea_warp.cuh"

namespace alea_gpu {

namespace {

constexpr double kTwoPiD = 6.283185307179586476925286766559;
constexpr double kInvTwoPiD = 0.15915494309189533576888376337251;

// sin, cos of an FP64 angle: reduced to [-π, π] in FP64, evaluated in FP32.
__device__ __forceinline__ void sincos_reduced(double ang, float& sn, float& c) {
    const double t = ang * kInvTwoPiD;
    const float a = static_cast<float>((t - rint(t)) * kTwoPiD);
    sincosf(a, &sn, &c);
}

// Orbital i of a real block at (x, y) in FP32 (angles and displacements in FP64).
__device__ __forceinline__ void orbital2f(const DevSys& s, const DevBlock& B, int i, double x, double y,
                                          float& val, float& gx, float& gy, float& lx, float& ly) {
    if (B.type == 0) {
        const double k0d = B.k[i * 2], k1d = B.k[i * 2 + 1];
        const float k0 = static_cast<float>(k0d), k1 = static_cast<float>(k1d);
        float sn, c;
        sincos_reduced(fma(k1d, y, k0d * x), sn, c);
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
        const float alpha = static_cast<float>(B.alphas[i]);
        double dxd = x - B.centers[i * 2], dyd = y - B.centers[i * 2 + 1];
        min_image2(s, dxd, dyd);
        const float dx = static_cast<float>(dxd), dy = static_cast<float>(dyd);
        const float phi = expf(-alpha * fmaf(dy, dy, dx * dx));
        val = phi;
        gx = phi * (-2.0f * alpha * dx);
        gy = phi * (-2.0f * alpha * dy);
        lx = phi * (4.0f * alpha * alpha * dx * dx - 2.0f * alpha);
        ly = phi * (4.0f * alpha * alpha * dy * dy - 2.0f * alpha);
    }
}

// The breakup spline in FP32 (coefficients read in FP64, rounded once).
__device__ __forceinline__ void spline3f(const DevSpline& sp, float r, float& f, float& df, float& d2f) {
    const float inv_delta = static_cast<float>(sp.inv_delta);
    const float t = r * inv_delta;
    int i = static_cast<int>(t);
    if (i > sp.n_knots - 2) i = sp.n_knots - 2;
    const float x = t - static_cast<float>(i);
    const double2* c2 = reinterpret_cast<const double2*>(sp.poly + 6 * i);
    const double2 c01 = ldg_keep(c2), c23 = ldg_keep(c2 + 1), c45 = ldg_keep(c2 + 2);
    const float a0 = static_cast<float>(c01.x), a1 = static_cast<float>(c01.y);
    const float a2 = static_cast<float>(c23.x), a3 = static_cast<float>(c23.y);
    const float a4 = static_cast<float>(c45.x), a5 = static_cast<float>(c45.y);
    f = fmaf(fmaf(fmaf(fmaf(fmaf(a5, x, a4), x, a3), x, a2), x, a1), x, a0);
    const float g = fmaf(fmaf(fmaf(fmaf(5.0f * a5, x, 4.0f * a4), x, 3.0f * a3), x, 2.0f * a2), x, a1);
    const float h = fmaf(fmaf(fmaf(20.0f * a5, x, 12.0f * a4), x, 6.0f * a3), x, 2.0f * a2);
    df = inv_delta * g;
    d2f = inv_delta * inv_delta * h;
}

// u, u', u'' of a Padé (kind 0) or Drummond (kind 1) pair term in FP32.
__device__ __forceinline__ void radial_pdf(const DevTerm& T, float r, float& u, float& du, float& d2u) {
    if (T.kind == 0) {
        float p = 0.0f, dp = 0.0f, d2p = 0.0f, q = 1.0f, dq = 0.0f, d2q = 0.0f;
        if (T.nnum == 1 && T.nden == 1) {
            const float a = static_cast<float>(T.coef[0]), b = static_cast<float>(T.coef[1]);
            p = a * r;
            dp = a;
            q = fmaf(b, r, 1.0f);
            dq = b;
        } else {
            float rk = 1.0f, rkm = 0.0f;
            for (int i = 0; i < T.nnum; ++i) {
                const float c = static_cast<float>(T.coef[i]);
                const int k = i + 1;
                p += c * rk * r;
                dp += c * static_cast<float>(k) * rk;
                d2p += c * static_cast<float>(k * (k - 1)) * rkm;
                rkm = rk;
                rk *= r;
            }
            rk = 1.0f;
            rkm = 0.0f;
            for (int i = 0; i < T.nden; ++i) {
                const float c = static_cast<float>(T.coef[T.nnum + i]);
                const int k = i + 1;
                q += c * rk * r;
                dq += c * static_cast<float>(k) * rk;
                d2q += c * static_cast<float>(k * (k - 1)) * rkm;
                rkm = rk;
                rk *= r;
            }
        }
        const float iq = 1.0f / q;
        u = p * iq;
        du = (dp * q - p * dq) * iq * iq;
        d2u = (d2p - (2.0f * dp * dq - 2.0f * p * dq * dq * iq + p * d2q) * iq) * iq;
        if (T.image) {
            if (r >= static_cast<float>(T.sp.r_cut)) {
                u = du = d2u = 0.0f;
                return;
            }
            float f, df, d2f;
            spline3f(T.sp, r, f, df, d2f);
            u -= static_cast<float>(T.u_inf) + f;
            du -= df;
            d2u -= d2f;
        }
        return;
    }
    const float t = r - static_cast<float>(T.L);
    float tCm2 = 1.0f;
    for (int i = 0; i < T.C - 2; ++i) tCm2 *= t;
    const float tCm1 = tCm2 * t, tC = tCm1 * t;
    const float g = tC, dg = static_cast<float>(T.C) * tCm1, d2g = static_cast<float>(T.C * (T.C - 1)) * tCm2;
    const float a1 = static_cast<float>(T.alpha1);
    float P = static_cast<float>(T.dc[0]) + a1 * r, dP = a1, d2P = 0.0f;
    float r_lm2 = 1.0f, r_lm1 = r, r_l = r * r;
    for (int k = 1; k < T.ncoef; ++k) {
        const int l = k + 1;
        const float c = static_cast<float>(T.dc[k]);
        P += c * r_l;
        dP += c * static_cast<float>(l) * r_lm1;
        d2P += c * static_cast<float>(l * (l - 1)) * r_lm2;
        r_lm2 = r_lm1;
        r_lm1 = r_l;
        r_l *= r;
    }
    const float m = (r < static_cast<float>(T.L)) ? 1.0f : 0.0f;
    u = m * (g * P);
    du = m * (dg * P + g * dP);
    d2u = m * (d2g * P + 2.0f * dg * dP + g * d2P);
}

// k-space terms of one k in FP32, added to FP64 sums.
__device__ __forceinline__ void kterm_f(float kx, float ky, float w, float c, float sn, float pr, float pi,
                                        float self, double* acc) {
    const float g = 2.0f * w * (c * pi - sn * pr);
    const float l = 2.0f * w * (self - (c * pr + sn * pi));
    acc[0] += static_cast<double>(kx * g);
    acc[1] += static_cast<double>(ky * g);
    acc[2] += static_cast<double>(kx * kx * l);
    acc[3] += static_cast<double>(ky * ky * l);
}

// A blocks of the compact layout between FP64 (as in the record) and FP32
// (packed at the start of each block's region), in 32-element chunks so that
// no lane overwrites a value another lane has still to read.
__device__ void blocks_to_f32(const DevSys& s, const Smem& v) {
    for (int b = 0; b < s.nblocks; ++b) {
        double* A = v.scal - s.o_scal + s.blocks[b].oA;
        float* Af = reinterpret_cast<float*>(A);
        const int n = s.blocks[b].n * s.blocks[b].n;
        for (int c0 = 0; c0 < n; c0 += 32) {
            const int i = c0 + static_cast<int>(threadIdx.x);
            const double x = i < n ? A[i] : 0.0;
            __syncwarp();
            if (i < n) Af[i] = static_cast<float>(x);
            __syncwarp();
        }
    }
}

__device__ void blocks_to_f64(const DevSys& s, const Smem& v) {
    for (int b = 0; b < s.nblocks; ++b) {
        double* A = v.scal - s.o_scal + s.blocks[b].oA;
        const float* Af = reinterpret_cast<const float*>(A);
        const int n = s.blocks[b].n * s.blocks[b].n;
        for (int c0 = (n - 1) / 32 * 32; c0 >= 0; c0 -= 32) {
            const int i = c0 + static_cast<int>(threadIdx.x);
            const float x = i < n ? Af[i] : 0.0f;
            __syncwarp();
            if (i < n) A[i] = static_cast<double>(x);
            __syncwarp();
        }
    }
}

// Full inverse recomputation of block b in FP64: the orbital rows at the
// current positions (the moved particle's row at (mx, my)) into `m`, then
// the in-place warp Gauss-Jordan of the FP64 sweep (gj_invert_warp, the
// reference's pivot rule); the inverse is rounded into the FP32 block.  log|det| to misc[M_LOGDET], a bad pivot to misc[M_ERR]; the
// row sums of |inverse| come back as the lane's maximum.
template <int S>
__device__ double rebuild_f64(const DevSys& s, const Smem& v, int b, int moved, double mx, double my) {
    const DevBlock& B = s.blocks[b];
    const int N = B.n;
    const int lane = threadIdx.x;
    double* m = v.work;
    float* Af = reinterpret_cast<float*>(v.scal - s.o_scal + B.oA);
    __syncwarp();
    for (int e = lane; e < N * N; e += 32) {
        const int r = e / N, c = e - r * N;
        const int part = B.first + r;
        const double x = part == moved ? mx : v.pos[part * 2], y = part == moved ? my : v.pos[part * 2 + 1];
        double val, gx, gy, lx, ly;
        orbital2(s, B, c, x, y, val, gx, gy, lx, ly);
        m[e] = val;
    }
    gj_invert_warp<S>(m, v.rowp, v.col, N, v.misc);
    double rs = 0.0;
    for (int r = lane; r < N; r += 32) {
        double t = 0.0;
        for (int c = 0; c < N; ++c) {
            const double x = m[r * N + c];
            Af[r * N + c] = static_cast<float>(x);
            t += fabs(x);
        }
        rs = fmax(rs, t);
    }
    __syncwarp();
    return rs;
}

// ρ(k) of every group from the positions, in FP64 (the FP32 changes of the
// moves are added to FP64 totals; the local energy starts from exact ones).
// Lane slot i walks the k list with its particle's phase; four k at a time
// the lanes' (Re, Im) for one group meet in an 8-value reduce-scatter.
template <int S>
__device__ void rho_from_positions(const DevSys& s, const Smem& v) {
    const int np = s.np, nk = s.nkJ;
    const int lane = threadIdx.x & 31;
    double th1[S], th2[S], e2r[S], e2i[S];
    int gi[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int i = lane + 32 * j;
        gi[j] = i < np ? s.group_of[i] : -1;
        const double x = i < np ? v.pos[i * 2] : 0.0, y = i < np ? v.pos[i * 2 + 1] : 0.0;
        th1[j] = s.recip[0] * x + s.recip[1] * y;
        th2[j] = s.recip[2] * x + s.recip[3] * y;
        sincos(th2[j], &e2i[j], &e2r[j]);
    }
    for (int g = 0; g < s.ngroups; ++g) {
        double c[S], sn[S];
        PhaseWalk walk[S];
#pragma unroll
        for (int j = 0; j < S; ++j) c[j] = 1.0, sn[j] = 0.0;
        for (int kb = 0; kb < nk; kb += 4) {
            double val[8];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int q = kb + t;
                double vr = 0.0, vi = 0.0;
                if (q < nk) {
                    const int m1 = s.n1J[q], m2 = s.n2J[q];
#pragma unroll
                    for (int j = 0; j < S; ++j) {
                        walk[j].next(m1, m2, th1[j], th2[j], e2r[j], e2i[j], c[j], sn[j]);
                        if (gi[j] == g) {
                            vr += c[j];
                            vi += sn[j];
                        }
                    }
                }
                val[2 * t] = vr;
                val[2 * t + 1] = vi;
            }
            const double tot = warp_reduce_scatter<8>(val);
            const int idx = lane >> 2;   // value idx: k offset idx >> 1, part idx & 1
            if ((lane & 3) == 0 && kb + (idx >> 1) < nk)
                v.rho[g * 2 * nk + (idx & 1) * nk + kb + (idx >> 1)] = tot;
        }
    }
    __syncwarp();
}

// The local energy after an FP32 sweep, in FP64: determinant derivatives from
// the FP32 inverse and FP64 orbital derivatives recomputed at the positions,
// ρ(k) recomputed, then the k-space refresh, kinetic, Ewald and pair
// potentials of the FP64 path.
template <int S>
__device__ __noinline__ double local_energy_f32(const DevSys& s, double* sm, const int2* pairs, int npair) {
    const Smem v = view_fast(s, sm, true);
    __syncwarp();
    for (int i = threadIdx.x; i < 2 * s.np; i += 32) v.sg[i] = v.sl[i] = v.kg[i] = v.kl[i] = 0.0;
    __syncwarp();
    for (int b = 0; b < s.nblocks; ++b) {
        const DevBlock& B = s.blocks[b];
        const int N = B.n;
        const float* Af = reinterpret_cast<const float*>(v.scal - s.o_scal + B.oA);
        for (int kr = threadIdx.x; kr < N; kr += 32) {
            const int part = B.first + kr;
            const double x = v.pos[part * 2], y = v.pos[part * 2 + 1];
            double g0 = 0.0, g1 = 0.0, l0 = 0.0, l1 = 0.0;
            for (int mo = 0; mo < N; ++mo) {
                double val, gx, gy, lx, ly;
                orbital2(s, B, mo, x, y, val, gx, gy, lx, ly);
                const double a = static_cast<double>(Af[mo * N + kr]);
                g0 += a * gx;
                g1 += a * gy;
                l0 += a * lx;
                l1 += a * ly;
            }
            v.sg[part * 2] = g0;
            v.sg[part * 2 + 1] = g1;
            v.sl[part * 2] = l0 - g0 * g0;
            v.sl[part * 2 + 1] = l1 - g1 * g1;
        }
    }
    if (s.nkJ > 0) {
        rho_from_positions<S>(s, v);
        kspace_refresh_warp<S>(s, v);
    }
    __syncwarp();
    return local_energy<32, S>(s, v, pairs, npair);
}

}  // namespace

template <int S>
__global__ void __launch_bounds__(32, 12) sweep_f32_kernel(const __grid_constant__ DevSys s, double* records,
                                                       int nw, const double* randoms, long stride,
                                                       SweepParams prm, const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    const int lane = threadIdx.x;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_fast(s, rec, sm);
    const Smem v = view_fast(s, sm, false);
    blocks_to_f32(s, v);
    const int np = s.np, nk = s.nkJ;
    const bool dmc = prm.mode == 1;
    const bool drift = dmc || prm.drift != 0;
    float* nvalf = reinterpret_cast<float*>(v.nval);    // new orbital row: value, ∇x, ∇y, ∂²x, ∂²y
    float* ngf = reinterpret_cast<float*>(v.ngrad);
    float* nlf = reinterpret_cast<float*>(v.nlap);
    float* colf = reinterpret_cast<float*>(v.col);
    float* rowpf = reinterpret_cast<float*>(v.rowp);
    float* cof = reinterpret_cast<float*>(v.co);        // p's phases and their changes
    float* sof = reinterpret_cast<float*>(v.so);
    float* dcf = reinterpret_cast<float*>(v.cn);
    float* dsf = reinterpret_cast<float*>(v.sn);
    float* djf = reinterpret_cast<float*>(v.work);      // partners' derivative changes
    int kgrp[S];
    unsigned long long cmask[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        const int k = lane + 32 * j;
        kgrp[j] = k < np ? s.group_of[k] : 0;
        unsigned long long msk = 0;
        if (k < np)
            for (int g = 0; g < s.ngroups; ++g)
                msk |= static_cast<unsigned long long>(s.gterms[g][kgrp[j]]) << (8 * g);
        cmask[j] = msk;
    }
    unsigned long long tgrp = 0;
    for (int t = 0; t < s.nterms; ++t) {
        const unsigned ga = static_cast<unsigned>(s.group_of[s.terms[t].pairs[0][0]]);
        const unsigned gb = static_cast<unsigned>(s.group_of[s.terms[t].pairs[0][2]]);
        tgrp |= static_cast<unsigned long long>((ga & 15u) | ((gb & 15u) << 4)) << (8 * t);
    }
    unsigned long long gimask = 0;
    for (int g = 0; g < s.ngroups; ++g)
        for (int t = 0; t < s.nterms; ++t)
            if (s.terms[t].image && in_term(s.terms[t], s.gfirst[g])) gimask |= 1ull << (8 * g + t);
    if (lane == 0) {
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
    __syncwarp();
    for (int sub = 0; sub < prm.n_sub; ++sub) {
        const double* rnd = randoms + static_cast<long>(sub) * np * 3 * stride;
        double rz0[S], rz1[S], rzu[S];
#pragma unroll
        for (int j = 0; j < S; ++j) {
            const int k = lane + 32 * j;
            const double* g = rnd + static_cast<long>(k) * 3 * stride + w;
            rz0[j] = k < np ? __ldcs(g) : 0.0;
            rz1[j] = k < np ? __ldcs(g + stride) : 0.0;
            rzu[j] = k < np ? __ldcs(g + 2 * stride) : 0.0;
        }
        for (int p = 0; p < np; ++p) {
            const int gp = from_owner<S>(kgrp, p);
            const int b = block_of(s, p);
            const unsigned imask = nk > 0 ? static_cast<unsigned>((gimask >> (8 * gp)) & 0xffu) : 0u;
            const bool ks = imask != 0;
            const double px = v.pos[p * 2], py = v.pos[p * 2 + 1];
            // ── drift refresh of p (FP32 terms, FP64 sums) ──
            double sgp0 = 0.0, sgp1 = 0.0, kgp0 = 0.0, kgp1 = 0.0;
            if (drift) {
                double ra[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // 0-1 determinant ∇, 4-7 k-space ∇, ∂²
                if (b >= 0) {
                    const DevBlock& B = s.blocks[b];
                    const int N = B.n, kr = p - B.first;
                    const float* Af = reinterpret_cast<const float*>(v.scal - s.o_scal + B.oA);
                    for (int m = lane; m < N; m += 32) {
                        float val, gx, gy, lx, ly;
                        orbital2f(s, B, m, px, py, val, gx, gy, lx, ly);
                        const float a = Af[m * N + kr];
                        ra[0] += static_cast<double>(a * gx);
                        ra[1] += static_cast<double>(a * gy);
                    }
                }
                if (ks) {
#pragma unroll 1
                    for (int q = lane; q < nk; q += 32) {
                        const double kxd = ldg_keep(s.kxJ + q), kyd = ldg_keep(s.kyJ + q);
                        const float kx = static_cast<float>(kxd), ky = static_cast<float>(kyd);
                        float co, so;
                        sincos_reduced(fma(kyd, py, kxd * px), so, co);
                        cof[q] = co;
                        sof[q] = so;
                        for (unsigned bits = imask; bits; bits &= bits - 1) {
                            const int t = __ffs(bits) - 1;
                            const DevTerm& T = s.terms[t];
                            const int ga = static_cast<int>((tgrp >> (8 * t)) & 15u);
                            const int gb = static_cast<int>((tgrp >> (8 * t + 4)) & 15u);
                            const int go = T.same0 ? gp : (gp == ga ? gb : ga);
                            const double* pr = v.rho + go * 2 * nk;
                            kterm_f(kx, ky, static_cast<float>(ldg_keep(T.kw + q)), co, so,
                                    static_cast<float>(pr[q]), static_cast<float>(pr[nk + q]),
                                    T.same0 ? 1.0f : 0.0f, ra + 4);
                        }
                    }
                }
                warp_allsum<8>(ra);
                sgp0 = b >= 0 ? ra[0] : 0.0;
                sgp1 = b >= 0 ? ra[1] : 0.0;
                kgp0 = ks ? ra[4] : 0.0;
                kgp1 = ks ? ra[5] : 0.0;
                __syncwarp();
            }
            // ── proposal (FP64, as the FP64 path) ──
            const double r0 = from_owner<S>(rz0, p), r1 = from_owner<S>(rz1, p), u = from_owner<S>(rzu, p);
            const double im0 = ldg_keep(s.inv_mass + p * 2), im1 = ldg_keep(s.inv_mass + p * 2 + 1);
            const double tm = prm.tau * im0;
            const double gx = sgp0 + v.jg[p * 2] + kgp0;
            const double gy = sgp1 + v.jg[p * 2 + 1] + kgp1;
            double sc = tm;
            if (dmc) {
                const double vsq = gx * gx + gy * gy;
                sc = vsq < 1e-10 ? tm : (-1.0 + sqrt(1.0 + 2.0 * tm * vsq)) / vsq;
            }
            const double sig0 = ldg_keep(prm.sigma + p * 2), sig1 = ldg_keep(prm.sigma + p * 2 + 1);
            double nx, ny;
            if (drift) {
                const double t0 = dmc ? sc : prm.tau * im0;
                const double t1 = dmc ? sc : prm.tau * im1;
                nx = fma(sig0, r0, fma(t0, gx, px));
                ny = fma(sig1, r1, fma(t1, gy, py));
            } else {
                nx = fma(sig0, r0, px);
                ny = fma(sig1, r1, py);
            }
            // ── ratio ──
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.0;
            if (b >= 0) {
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                const float* Af = reinterpret_cast<const float*>(v.scal - s.o_scal + B.oA);
#pragma unroll 1
                for (int m = lane; m < N; m += 32) {
                    float val, ogx, ogy, olx, oly;
                    orbital2f(s, B, m, nx, ny, val, ogx, ogy, olx, oly);
                    nvalf[m] = val;
                    ngf[m * 2 + 0] = ogx;
                    ngf[m * 2 + 1] = ogy;
                    nlf[m * 2 + 0] = olx;
                    nlf[m * 2 + 1] = oly;
                    const float a = Af[m * N + jrow];
                    const float term = a * val;
                    acc[0] += static_cast<double>(term);
                    acc[1] += static_cast<double>(fabsf(term));
                    acc[2] += static_cast<double>(a * ogx);
                    acc[3] += static_cast<double>(a * ogy);
                    acc[4] += static_cast<double>(a * olx);
                    acc[5] += static_cast<double>(a * oly);
                    acc[15] += static_cast<double>(fabsf(val));
                }
            }
            {
                unsigned cm[S];
                float rn[S], ro[S], dnx[S], dny[S], dox[S], doy[S];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    const int k = lane + 32 * j;
                    cm[j] = (k < np && k != p) ? static_cast<unsigned>((cmask[j] >> (8 * gp)) & 0xffu) : 0u;
                    const double kx0 = cm[j] ? v.pos[k * 2] : px + 1.0;
                    const double ky0 = cm[j] ? v.pos[k * 2 + 1] : py;
                    double a0, a1, b0, b1;
                    const double rnd_ = fold2(s, nx, ny, kx0, ky0, a0, a1);
                    const double rod_ = fold2(s, px, py, kx0, ky0, b0, b1);
                    rn[j] = cm[j] ? static_cast<float>(rnd_) : 1.0f;
                    ro[j] = cm[j] ? static_cast<float>(rod_) : 1.0f;
                    dnx[j] = static_cast<float>(a0);
                    dny[j] = static_cast<float>(a1);
                    dox[j] = static_cast<float>(b0);
                    doy[j] = static_cast<float>(b1);
                }
                float uo[S], duo[S], d2uo[S], un[S], dun[S], d2un[S];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    const DevTerm& T = s.terms[cm[j] ? __ffs(cm[j]) - 1 : 0];
                    radial_pdf(T, ro[j], uo[j], duo[j], d2uo[j]);
                    radial_pdf(T, rn[j], un[j], dun[j], d2un[j]);
                }
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    for (unsigned bits = cm[j] & (cm[j] - 1); bits; bits &= bits - 1) {
                        const DevTerm& T = s.terms[__ffs(bits) - 1];
                        float a0, a1, a2, b0, b1, b2;
                        radial_pdf(T, ro[j], a0, a1, a2);
                        radial_pdf(T, rn[j], b0, b1, b2);
                        uo[j] += a0;
                        duo[j] += a1;
                        d2uo[j] += a2;
                        un[j] += b0;
                        dun[j] += b1;
                        d2un[j] += b2;
                    }
                }
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    if (!cm[j]) continue;
                    const float irn = 1.0f / rn[j], iro = 1.0f / ro[j];
                    acc[6] += static_cast<double>(un[j] - uo[j]);
                    float* dj = djf + (lane + 32 * j) * 4;
                    {
                        const float dor = dnx[j] * irn;
                        acc[7] += static_cast<double>(dun[j] * dor);
                        acc[9] += static_cast<double>(d2un[j] * dor * dor + dun[j] * irn * (1.0f - dor * dor));
                        const float dor_old = -dox[j] * iro, dor_new = -dnx[j] * irn;
                        dj[0] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[2] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0f - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0f - dor_old * dor_old));
                    }
                    {
                        const float dor = dny[j] * irn;
                        acc[8] += static_cast<double>(dun[j] * dor);
                        acc[10] += static_cast<double>(d2un[j] * dor * dor + dun[j] * irn * (1.0f - dor * dor));
                        const float dor_old = -doy[j] * iro, dor_new = -dny[j] * irn;
                        dj[1] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[3] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0f - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0f - dor_old * dor_old));
                    }
                }
            }
            if (ks) {
#pragma unroll 1
                for (int q = lane; q < nk; q += 32) {
                    const double kxd = ldg_keep(s.kxJ + q), kyd = ldg_keep(s.kyJ + q);
                    const float kx = static_cast<float>(kxd), ky = static_cast<float>(kyd);
                    float cn, sn, co, so;
                    sincos_reduced(fma(kyd, ny, kxd * nx), sn, cn);
                    if (drift) {
                        co = cof[q];
                        so = sof[q];
                    } else {
                        sincos_reduced(fma(kyd, py, kxd * px), so, co);
                    }
                    const double* mr = v.rho + gp * 2 * nk;
                    const float dc = cn - co, ds = sn - so;
                    for (unsigned bits = imask; bits; bits &= bits - 1) {
                        const int t = __ffs(bits) - 1;
                        const DevTerm& T = s.terms[t];
                        const float wk = static_cast<float>(ldg_keep(T.kw + q));
                        if (T.same0) {
                            const float mrr = static_cast<float>(mr[q]), mri = static_cast<float>(mr[nk + q]);
                            const float qr = mrr + dc, qi = mri + ds;
                            // |ρ + δ|² - |ρ|² = δ·(2ρ + δ), without the cancellation
                            acc[6] += static_cast<double>(wk * (dc * (2.0f * mrr + dc) + ds * (2.0f * mri + ds)));
                            kterm_f(kx, ky, wk, cn, sn, qr, qi, 1.0f, acc + 11);
                        } else {
                            const int ga = static_cast<int>((tgrp >> (8 * t)) & 15u);
                            const int gb = static_cast<int>((tgrp >> (8 * t + 4)) & 15u);
                            const int go = gp == ga ? gb : ga;
                            const double* orr = v.rho + go * 2 * nk;
                            const float orr_r = static_cast<float>(orr[q]), orr_i = static_cast<float>(orr[nk + q]);
                            acc[6] += static_cast<double>(2.0f * wk * (dc * orr_r + ds * orr_i));
                            kterm_f(kx, ky, wk, cn, sn, orr_r, orr_i, 0.0f, acc + 11);
                        }
                    }
                    dcf[q] = dc;
                    dsf[q] = ds;
                }
            }
            warp_allsum<16>(acc);
            double logr = acc[6], phase = 0.0, logdr = 0.0, sgx = 0.0, sgy = 0.0;
            if (b >= 0) {
                const double R = acc[0];
                logdr = log(fmax(fabs(R), 1e-300));
                if (R < 0.0) phase = kPi;
                const double invR = (R != 0.0) ? 1.0 / R : 0.0;
                sgx = invR * acc[2];
                sgy = invR * acc[3];
            }
            logr += logdr;
            const double ngx_t = sgx + acc[7] + acc[11], ngy_t = sgy + acc[8] + acc[12];
            const double dx = nx - px, dy = ny - py;
            const double tm0 = prm.tau * im0, tm1 = prm.tau * im1;
            bool accept;
            if (dmc) {
                accept = false;
                if (phase == 0.0) {
                    const double vsq = ngx_t * ngx_t + ngy_t * ngy_t;
                    const double sb = vsq < 1e-10 ? tm0 : (-1.0 + sqrt(1.0 + 2.0 * tm0 * vsq)) / vsq;
                    double lc = 0.0;
                    if (tm0 > 0.0) {
                        const double df = sc * gx, db = sb * ngx_t;
                        lc += (-dx * (df + db) + 0.5 * (df * df - db * db)) / tm0;
                    }
                    if (tm1 > 0.0) {
                        const double df = sc * gy, db = sb * ngy_t;
                        lc += (-dy * (df + db) + 0.5 * (df * df - db * db)) / tm1;
                    }
                    const double la = 2.0 * logr + lc;
                    accept = la >= 0.0 || u < exp(la);
                }
                if (lane == 0) {
                    const double rr = tm0 * dx * dx + tm1 * dy * dy;
                    v.scal[S_RRP] += rr;
                    if (accept) v.scal[S_RRA] += rr;
                }
            } else if (prm.drift) {
                double lc = -dx * (gx + ngx_t) + 0.5 * tm0 * (gx * gx - ngx_t * ngx_t);
                lc += -dy * (gy + ngy_t) + 0.5 * tm1 * (gy * gy - ngy_t * ngy_t);
                const double la = 2.0 * logr + lc;
                accept = la >= 0.0 || u < exp(la);
            } else {
                accept = u < exp(2.0 * logr);
            }
            if (!accept) continue;
            // ── commit ──
            if (lane == 0) v.scal[S_NACC] += 1.0;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                const int k = lane + 32 * j;
                if (k >= np || k == p || ((cmask[j] >> (8 * gp)) & 0xffu) == 0) continue;
                const float* dj = djf + k * 4;
                v.jg[k * 2 + 0] += static_cast<double>(dj[0]);
                v.jg[k * 2 + 1] += static_cast<double>(dj[1]);
                v.jl[k * 2 + 0] += static_cast<double>(dj[2]);
                v.jl[k * 2 + 1] += static_cast<double>(dj[3]);
            }
            if (ks) {
                double* mr = v.rho + gp * 2 * nk;
                for (int q = lane; q < nk; q += 32) {
                    mr[q] += static_cast<double>(dcf[q]);
                    mr[nk + q] += static_cast<double>(dsf[q]);
                }
            }
            if (b >= 0) {
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                float* Af = reinterpret_cast<float*>(v.scal - s.o_scal + B.oA);
                double* bs = v.scal + S_BLOCK0 + 3 * b;
                double* rabs = v.scal - s.o_scal + B.orabs;
                const double R = acc[0];
                const float Rf = static_cast<float>(R);
                __syncwarp();   // the new orbital row
#pragma unroll 1
                for (int c = lane; c < N; c += 32) {
                    float pa = 0.0f, pb = 0.0f;
                    int m = 0;
                    for (; m + 1 < N; m += 2) {
                        pa = fmaf(nvalf[m], Af[m * N + c], pa);
                        pb = fmaf(nvalf[m + 1], Af[(m + 1) * N + c], pb);
                    }
                    if (m < N) pa = fmaf(nvalf[m], Af[m * N + c], pa);
                    rowpf[c] = (pa + pb) - (c == jrow ? 1.0f : 0.0f);
                    colf[c] = Af[c * N + jrow] / Rf;
                }
                const double upd = bs[1] + 1.0;
                const double old_log = bs[0];
                bool rebuild = upd >= 64.0 || !isfinite(R) || fabs(R) < 1e-5 || bs[2] > 1e8 ||
                               fabs(R) <= 1e4 * kEps * acc[1];
                __syncwarp();
                if (lane == 0) {
                    bs[1] = upd;
                    rabs[jrow] = acc[15];
                }
                double rs_max = 0.0, rd_max = 0.0;
                if (!rebuild) {
#pragma unroll 1
                    for (int a = lane; a < N; a += 32) {
                        const float ca = colf[a];
                        float ra = 0.0f, rb = 0.0f;
                        int c = 0;
                        for (; c + 1 < N; c += 2) {
                            const float x0 = fmaf(-ca, rowpf[c], Af[a * N + c]);
                            const float x1 = fmaf(-ca, rowpf[c + 1], Af[a * N + c + 1]);
                            Af[a * N + c] = x0;
                            Af[a * N + c + 1] = x1;
                            ra += fabsf(x0);
                            rb += fabsf(x1);
                        }
                        if (c < N) {
                            const float x0 = fmaf(-ca, rowpf[c], Af[a * N + c]);
                            Af[a * N + c] = x0;
                            ra += fabsf(x0);
                        }
                        rs_max = fmax(rs_max, static_cast<double>(ra + rb));
                    }
                }
                __syncwarp();
                for (int a = lane; a < N; a += 32) rd_max = fmax(rd_max, rabs[a]);
                rd_max = warp_max(rd_max);
                double cond = rebuild ? 0.0 : rd_max * warp_max(rs_max);
                const bool cond_rebuild = !rebuild && (!isfinite(cond) || cond > 1e8);
                if (__builtin_expect(rebuild || cond_rebuild, 0)) {
                    const double rs = rebuild_f64<S>(s, v, b, p, nx, ny);
                    if (rebuild) cond = rd_max * warp_max(rs);
                    rebuild = true;
                }
                if (lane == 0) {
                    bs[2] = cond;
                    if (rebuild) {
                        bs[0] = v.misc[M_LOGDET];
                        bs[1] = 0.0;
                        if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
                    } else {
                        bs[0] = old_log + log(fabs(R));
                    }
                    v.scal[S_LOGPSI] += bs[0] - old_log;
                }
            }
            if (lane == 0) {
                v.jg[p * 2 + 0] = acc[7];
                v.jg[p * 2 + 1] = acc[8];
                v.jl[p * 2 + 0] = acc[9];
                v.jl[p * 2 + 1] = acc[10];
                double wx = nx, wy = ny;
                wrap2(s, wx, wy);
                v.pos[p * 2 + 0] = wx;
                v.pos[p * 2 + 1] = wy;
                v.scal[S_LOGPSI] += logr - logdr;
            }
            __syncwarp();
        }
        if (dmc || sub == prm.n_sub - 1) {
            __syncwarp();
            const double el = local_energy_f32<S>(s, sm, pairs, npair);
            if (lane == 0) {
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
            __syncwarp();
        }
    }
    if (lane == 0) {
        if (dmc && prm.tau > 0.0) v.scal[S_AGE] = v.scal[S_RRP] > 0.0 ? 0.0 : v.scal[S_AGE] + 1.0;
        if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
    }
    __syncwarp();
    blocks_to_f64(s, v);
    store_fast(s, rec, sm);
}

// Plane-wave determinants only: localized Gaussian orbitals make D too badly
// conditioned for FP32 rank-one updates (a 16-particle crystal's local
// energies drifted by 4e-5 Ha per particle within a few sweeps, above the
// 1e-5 bound the form is held to).
bool f32_sweep_eligible(const DevSys& s) {
    if (!fast_sweep_eligible(s)) return false;
    for (int t = 0; t < s.nterms; ++t)
        if (s.terms[t].kind == 2) return false;   // the zero-energy form has no FP32 restatement
    for (int b = 0; b < s.nblocks; ++b)
        if (s.blocks[b].type != 0) return false;
    return true;
}

cudaError_t reserve_smem_f32(size_t smem) {
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(sweep_f32_kernel<2>),
                                cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
}

cudaError_t launch_sweep_f32(int nw, cudaStream_t st, const DevSys& s, double* records, const double* randoms,
                             long stride, const SweepParams& prm, const int2* pairs, int npair) {
    sweep_f32_kernel<2><<<nw, 32, static_cast<size_t>(s.f_total32) * 8, st>>>(s, records, nw, randoms, stride,
                                                                            prm, pairs, npair);
    return cudaGetLastError();
}

}  // namespace alea_gpu
