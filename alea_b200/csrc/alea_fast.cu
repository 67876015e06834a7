// The one-warp VMC/DMC sweep (sm_100a) for systems of real determinants and
// pair Jastrows of at most 64 particles: one CTA of 32 threads per walker,
// the walker's hot state in shared memory as in the generic sweep, and every
// per-item intermediate of a move in registers.
//
// Algorithms restated from the reference (ItaloAlb/alea), in the same steps
// as the generic sweep of alea_kernels.cu:
//   sweep          src/qmc/vmc.cpp:82-155, src/qmc/dmc.cpp:203-337,
//                  src/numerics/green_function.h:20-58
//   Slater         src/wavefunction/slater_determinant.cpp:395-437 (ratio),
//                  :515-726 (Sherman-Morrison commit, rebuild triggers),
//                  :862-903 (derivative refresh), :905-993 (Gauss-Jordan)
//   pair Jastrows  src/wavefunction/pade_jastrow.cpp:347-634,
//                  src/wavefunction/radial_pair_jastrow_impl.h
//   image sums     src/wavefunction/kspace_pair_sum.cpp:157-301
//   E_L, weights   src/hamiltonian/kinetic.cpp:45-72, ewald_term.cpp:368-612,
//                  src/qmc/population_control.cpp:56-77
//
// Work split.  Lane l owns slot j = 0..S-1 of every list: partner l + 32j
// (its displacement, radial terms and its own Jastrow-derivative change,
// applied by the same lane if the move is accepted), orbital row l + 32j
// (new orbital value and derivatives, its factor of the rank-one update, its
// rows of D, ∇D, ∇²D written back), k-vector l + 32j (old and new phase, the
// change of ρ(k)).  The per-move sums (ratio, ∇ and ∂² of the moved particle,
// log J) meet in one 16-value warp reduce-scatter; every lane ends with the
// same totals and takes the accept decision itself, so a move has no block
// barrier.  The orbital rows of the next particle are fetched from HBM while
// the current move runs, and a sweep's random numbers are read once per lane.
#include "alea_warp.cuh"

namespace alea_gpu {

// One walker's sweep by one warp (the body of sweep_fast_kernel and of the
// packed launches).  C: the determinants are complex (twisted plane waves,
// complex_slater_determinant.cpp:154-256): orbital values are recomputed
// from the positions (one sincos per orbital) instead of read from stored
// rows, the inverse is re | im, the update is the complex rank-one form and
// the refresh after 64 updates a complex Gauss-Jordan; the fixed-phase DMC
// accept has no node gate.
template <int S, bool ZE, bool C>
__device__ __forceinline__ void sweep_fast_walker(const DevSys& s, double* records, int w, const double* randoms,
                                                  long stride, const SweepParams& prm, const int2* pairs,
                                                  int npair, double* sm) {
    const int lane = threadIdx.x;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_fast(s, rec, sm);
    const Smem v = view_fast(s, sm, false);
    const int np = s.np, nk = s.nkJ;
    const bool dmc = prm.mode == 1;
    const bool drift = dmc || prm.drift != 0;
    // partner slots: group, and the terms coupling the partner to each group
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
    // groups of each term's first pair, 4 bits each: byte t = ga | gb << 4
    unsigned long long tgrp = 0;
    for (int t = 0; t < s.nterms; ++t) {
        const unsigned ga = static_cast<unsigned>(s.group_of[s.terms[t].pairs[0][0]]);
        const unsigned gb = static_cast<unsigned>(s.group_of[s.terms[t].pairs[0][2]]);
        tgrp |= static_cast<unsigned long long>((ga & 15u) | ((gb & 15u) << 4)) << (8 * t);
    }
    // image-summed terms each group takes part in (bit t of byte g)
    unsigned long long gimask = 0;
    for (int g = 0; g < s.ngroups; ++g)
        for (int t = 0; t < s.nterms; ++t)
            if (s.terms[t].image && in_term(s.terms[t], s.gfirst[g]))
                gimask |= 1ull << (8 * g + t);
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
        double2 dg[S], dl[S];
#pragma unroll
        for (int j = 0; j < S; ++j) dg[j] = dl[j] = make_double2(0.0, 0.0);
        if (!C && drift) fetch_rows<S>(s, rec, 0, dg, dl);
        for (int p = 0; p < np; ++p) {
            const int gp = from_owner<S>(kgrp, p);
            const int b = block_of(s, p);
            const unsigned imask = nk > 0 ? static_cast<unsigned>((gimask >> (8 * gp)) & 0xffu) : 0u;
            const bool ks = imask != 0;
            const double px = v.pos[p * 2], py = v.pos[p * 2 + 1];
            // ── drift refresh of p: determinant and k-space derivatives ──
            double sgp0 = 0.0, sgp1 = 0.0, kgp0 = 0.0, kgp1 = 0.0;
            if (drift) {
                double ra[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                if (C && b >= 0) {
                    // Re Σ_m A[m][kr] ∇φ_m(r_p), ∇φ = i q φ
                    const DevBlock& B = s.blocks[b];
                    const int N = B.n, kr = p - B.first;
                    const double* Ar = v.scal - s.o_scal + B.oA;
                    const double* Ai = Ar + ((N * N + 3) & ~3);
#pragma unroll 1
                    for (int m = lane; m < N; m += 32) {
                        const double qx = B.k[m * 2], qy = B.k[m * 2 + 1];
                        double sn, cs;
                        sincos(fma(qy, py, qx * px), &sn, &cs);
                        const double ti = Ar[m * N + kr] * sn + Ai[m * N + kr] * cs;
                        ra[0] += -qx * ti;
                        ra[1] += -qy * ti;
                    }
                } else if (b >= 0) {
                    const DevBlock& B = s.blocks[b];
                    const int N = B.n, kr = p - B.first;
                    const double* A = v.scal - s.o_scal + B.oA;
#pragma unroll
                    for (int j = 0; j < S; ++j) {
                        const int m = lane + 32 * j;
                        if (m >= N) continue;
                        const double a = A[m * N + kr];
                        ra[0] += a * dg[j].x;
                        ra[1] += a * dg[j].y;
                        ra[2] += a * dl[j].x;
                        ra[3] += a * dl[j].y;
                    }
                }
                if (!C && p + 1 < np) fetch_rows<S>(s, rec, p + 1, dg, dl);
                if (ks) {
#pragma unroll 1
                    for (int q = lane; q < nk; q += 32) {
                        const double kxq = ldg_keep(s.kxJ + q), kyq = ldg_keep(s.kyJ + q);
                        double co, so;
                        sincos(fma(kyq, py, kxq * px), &so, &co);
                        v.co[q] = co;
                        v.so[q] = so;
                        for (unsigned bits = imask; bits; bits &= bits - 1) {
                            const int t = __ffs(bits) - 1;
                            const DevTerm& T = s.terms[t];
                            const int ga = static_cast<int>((tgrp >> (8 * t)) & 15u);
                            const int gb = static_cast<int>((tgrp >> (8 * t + 4)) & 15u);
                            const int go = T.same0 ? gp : (gp == ga ? gb : ga);
                            const double* pr = v.rho + go * 2 * nk;
                            kterm_r(kxq, kyq, ldg_keep(T.kw + q), co, so, pr[q], pr[nk + q], T.same0 ? 1.0 : 0.0,
                                    ra + 4);
                        }
                    }
                }
                warp_allsum<8>(ra);
                sgp0 = ra[0];
                sgp1 = ra[1];
                kgp0 = ra[4];
                kgp1 = ra[5];
                __syncwarp();
            }
            // ── proposal (every lane, identical arithmetic) ──
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
            // acc: 0 R, 1 Σ|A φ|, 2-3 Σ A ∇φ, 4-5 Σ A ∂²φ, 6 log J, 7-8 pair ∇,
            // 9-10 pair ∂², 11-12 k-space ∇, 13-14 k-space ∂², 15 Σ|φ(r')|;
            // complex: 0-1 Re, Im R, 2-3 Re Σ A ∇φ, 4-5 Im Σ A ∇φ
            double acc[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) acc[i] = 0.0;
            if (C && b >= 0) {
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                const double* Ar = v.scal - s.o_scal + B.oA;
                const double* Ai = Ar + ((N * N + 3) & ~3);
#pragma unroll 1
                for (int m = lane; m < N; m += 32) {
                    const double qx = B.k[m * 2], qy = B.k[m * 2 + 1];
                    double sn, cs;
                    sincos(fma(qy, ny, qx * nx), &sn, &cs);
                    v.nval[m] = cs;
                    v.nval[N + m] = sn;
                    const double ar = Ar[m * N + jrow], ai = Ai[m * N + jrow];
                    const double tr = ar * cs - ai * sn, ti = ar * sn + ai * cs;
                    acc[0] += tr;
                    acc[1] += ti;
                    acc[2] += -qx * ti;
                    acc[3] += -qy * ti;
                    acc[4] += qx * tr;
                    acc[5] += qy * tr;
                }
            } else if (b >= 0) {
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                const double* A = v.scal - s.o_scal + B.oA;
#pragma unroll 1
                for (int m = lane; m < N; m += 32) {
                    double val, ogx, ogy, olx, oly;
                    orbital2(s, B, m, nx, ny, val, ogx, ogy, olx, oly);
                    v.nval[m] = val;
                    v.ngrad[m * 2 + 0] = ogx;
                    v.ngrad[m * 2 + 1] = ogy;
                    v.nlap[m * 2 + 0] = olx;
                    v.nlap[m * 2 + 1] = oly;
                    const double a = A[m * N + jrow];
                    const double term = a * val;
                    acc[0] += term;
                    acc[1] += fabs(term);
                    acc[2] += a * ogx;
                    acc[3] += a * ogy;
                    acc[4] += a * olx;
                    acc[5] += a * oly;
                    acc[15] += fabs(val);
                }
            }
            // pair terms: p's new derivatives, the log ratio, and each
            // partner's derivative change (kept in `work`, applied on accept).
            // Both partner slots go through each stage together so that their
            // four radial evaluations overlap; an idle slot runs on a dummy
            // partner at unit distance and contributes nothing.
            {
                unsigned cm[S];
                double rn[S], ro[S], dnx[S], dny[S], dox[S], doy[S];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    const int k = lane + 32 * j;
                    cm[j] = (k < np && k != p) ? static_cast<unsigned>((cmask[j] >> (8 * gp)) & 0xffu) : 0u;
                    const double kx0 = cm[j] ? v.pos[k * 2] : px + 1.0;
                    const double ky0 = cm[j] ? v.pos[k * 2 + 1] : py;
                    rn[j] = fold2(s, nx, ny, kx0, ky0, dnx[j], dny[j]);
                    ro[j] = fold2(s, px, py, kx0, ky0, dox[j], doy[j]);
                    if (!cm[j]) rn[j] = ro[j] = 1.0;
                }
                double uo[S], duo[S], d2uo[S], un[S], dun[S], d2un[S];
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    const DevTerm& T = s.terms[cm[j] ? __ffs(cm[j]) - 1 : 0];
                    radial_w<ZE>(T, ro[j], uo[j], duo[j], d2uo[j]);
                    radial_w<ZE>(T, rn[j], un[j], dun[j], d2un[j]);
                }
#pragma unroll
                for (int j = 0; j < S; ++j) {
                    // further terms on the same pair (rare)
                    for (unsigned bits = cm[j] & (cm[j] - 1); bits; bits &= bits - 1) {
                        const DevTerm& T = s.terms[__ffs(bits) - 1];
                        double a0, a1, a2, b0, b1, b2;
                        radial_w<ZE>(T, ro[j], a0, a1, a2);
                        radial_w<ZE>(T, rn[j], b0, b1, b2);
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
                    const double irn = 1.0 / rn[j], iro = 1.0 / ro[j];
                    acc[6] += un[j] - uo[j];
                    double* dj = v.work + (lane + 32 * j) * 4;
                    {
                        const double dor = dnx[j] * irn;
                        acc[7] += dun[j] * dor;
                        acc[9] += d2un[j] * dor * dor + dun[j] * irn * (1.0 - dor * dor);
                        const double dor_old = -dox[j] * iro, dor_new = -dnx[j] * irn;
                        dj[0] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[2] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0 - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0 - dor_old * dor_old));
                    }
                    {
                        const double dor = dny[j] * irn;
                        acc[8] += dun[j] * dor;
                        acc[10] += d2un[j] * dor * dor + dun[j] * irn * (1.0 - dor * dor);
                        const double dor_old = -doy[j] * iro, dor_new = -dny[j] * irn;
                        dj[1] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[3] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0 - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0 - dor_old * dor_old));
                    }
                }
            }
            // image sums: new phases of p, ratio and derivative terms; the
            // change of p's phases is kept in cn/sn for the ρ(k) update
            if (ks) {
#pragma unroll 1
                for (int q = lane; q < nk; q += 32) {
                    const double kxq = ldg_keep(s.kxJ + q), kyq = ldg_keep(s.kyJ + q);
                    double cn, sn, co, so;
                    sincos(fma(kyq, ny, kxq * nx), &sn, &cn);
                    if (drift) {
                        co = v.co[q];
                        so = v.so[q];
                    } else {
                        sincos(fma(kyq, py, kxq * px), &so, &co);
                    }
                    const double* mr = v.rho + gp * 2 * nk;
                    for (unsigned bits = imask; bits; bits &= bits - 1) {
                        const int t = __ffs(bits) - 1;
                        const DevTerm& T = s.terms[t];
                        const double wk = ldg_keep(T.kw + q);
                        if (T.same0) {
                            const double qr = mr[q] + cn - co;
                            const double qi = mr[nk + q] + sn - so;
                            acc[6] += wk * (qr * qr + qi * qi - mr[q] * mr[q] - mr[nk + q] * mr[nk + q]);
                            kterm_r(kxq, kyq, wk, cn, sn, qr, qi, 1.0, acc + 11);
                        } else {
                            const int ga = static_cast<int>((tgrp >> (8 * t)) & 15u);
                            const int gb = static_cast<int>((tgrp >> (8 * t + 4)) & 15u);
                            const int go = gp == ga ? gb : ga;
                            const double* orr = v.rho + go * 2 * nk;
                            acc[6] += 2.0 * wk * ((cn - co) * orr[q] + (sn - so) * orr[nk + q]);
                            kterm_r(kxq, kyq, wk, cn, sn, orr[q], orr[nk + q], 0.0, acc + 11);
                        }
                    }
                    v.cn[q] = cn - co;
                    v.sn[q] = sn - so;
                }
            }
            warp_allsum<16>(acc);
            double logr = acc[6], phase = 0.0, logdr = 0.0, sgx = 0.0, sgy = 0.0;
            if (C && b >= 0) {
                // |R| and Re(Σ A ∇φ / R); the phase of R moves no fixed-phase decision
                const double rr = acc[0], ri = acc[1];
                const double a2 = rr * rr + ri * ri;
                logdr = log(fmax(sqrt(a2), 1e-300));
                const double ir = a2 > 0.0 ? rr / a2 : 0.0, ii = a2 > 0.0 ? -ri / a2 : 0.0;
                sgx = acc[2] * ir - acc[4] * ii;
                sgy = acc[3] * ir - acc[5] * ii;
            } else if (b >= 0) {
                const double R = acc[0];
                logdr = log(fmax(fabs(R), 1e-300));
                if (R < 0.0) phase = kPi;
                const double invR = (R != 0.0) ? 1.0 / R : 0.0;
                sgx = invR * acc[2];
                sgy = invR * acc[3];
            }
            logr += logdr;
            // ── accept / reject (every lane, identical decision) ──
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
                const double* dj = v.work + k * 4;
                v.jg[k * 2 + 0] += dj[0];
                v.jg[k * 2 + 1] += dj[1];
                v.jl[k * 2 + 0] += dj[2];
                v.jl[k * 2 + 1] += dj[3];
            }
            if (ks) {
                double* mr = v.rho + gp * 2 * nk;
                for (int q = lane; q < nk; q += 32) {
                    mr[q] += v.cn[q];
                    mr[nk + q] += v.sn[q];
                }
            }
            if (C && b >= 0) {
                // complex Sherman-Morrison: A -= (A[:, j] / R) ⊗ (φ(r')ᵀ A - e_j),
                // Gauss-Jordan from the positions after 64 updates or at a
                // small or nonfinite ratio (the generic sweep's triggers)
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                double* Ar = v.scal - s.o_scal + B.oA;
                double* Ai = Ar + ((N * N + 3) & ~3);
                double* bs = v.scal + S_BLOCK0 + 3 * b;
                const double rr = acc[0], ri = acc[1];
                const double a2 = rr * rr + ri * ri;
                const double ir = rr / a2, ii = -ri / a2;
                const double* nr = v.nval;
                const double* ni = v.nval + N;
                __syncwarp();   // the new orbital row v.nval
#pragma unroll 1
                for (int c = lane; c < N; c += 32) {
                    double pr = 0.0, pi = 0.0;
                    for (int m = 0; m < N; ++m) {
                        const double xr = nr[m], xi = ni[m], ar = Ar[m * N + c], ai = Ai[m * N + c];
                        pr += xr * ar - xi * ai;
                        pi += xr * ai + xi * ar;
                    }
                    v.rowp[c] = pr - (c == jrow ? 1.0 : 0.0);
                    v.rowp[N + c] = pi;
                    const double cr = Ar[c * N + jrow], ci = Ai[c * N + jrow];
                    v.col[c] = cr * ir - ci * ii;
                    v.col[N + c] = cr * ii + ci * ir;
                }
                const double upd = bs[1] + 1.0;
                const double old_log = bs[0];
                const bool rebuild = upd >= 64.0 || !isfinite(a2) || sqrt(a2) < 1e-5;
                __syncwarp();
                if (!rebuild) {
#pragma unroll 1
                    for (int a = lane; a < N; a += 32) {
                        const double fr = v.col[a], fi = v.col[N + a];
                        for (int c = 0; c < N; ++c) {
                            const double qr = v.rowp[c], qi = v.rowp[N + c];
                            Ar[a * N + c] -= fr * qr - fi * qi;
                            Ai[a * N + c] -= fr * qi + fi * qr;
                        }
                    }
                } else {
                    cgj_rebuild_warp<S>(B, v.pos, p, nx, ny, Ar, Ai, v.work, v.col, v.misc);
                }
                __syncwarp();
                if (lane == 0) {
                    if (rebuild) {
                        bs[0] = v.misc[M_LOGDET];
                        bs[1] = 0.0;
                        if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
                    } else {
                        bs[0] = old_log + logdr;
                        bs[1] = upd;
                    }
                    v.scal[S_LOGPSI] += bs[0] - old_log;
                }
            } else if (b >= 0) {
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                double* A = v.scal - s.o_scal + B.oA;
                double* bs = v.scal + S_BLOCK0 + 3 * b;
                double* D = rec + B.oD;
                double2* Dg = reinterpret_cast<double2*>(rec + B.oDg) + jrow * N;
                double2* Dl = reinterpret_cast<double2*>(rec + B.oDl) + jrow * N;
                double* rabs = v.scal - s.o_scal + B.orabs;
                const double R = acc[0];
                const double inv_r = 1.0 / R;
                __syncwarp();   // the new orbital row v.nval
#pragma unroll 1
                for (int c = lane; c < N; c += 32) {
                    double pa = 0.0, pb = 0.0;
                    int m = 0;
                    for (; m + 1 < N; m += 2) {
                        pa += v.nval[m] * A[m * N + c];
                        pb += v.nval[m + 1] * A[(m + 1) * N + c];
                    }
                    if (m < N) pa += v.nval[m] * A[m * N + c];
                    v.rowp[c] = (pa + pb) - (c == jrow ? 1.0 : 0.0);
                    v.col[c] = A[c * N + jrow] * inv_r;   // factor of row c of the update
                    __stcg(D + jrow * N + c, v.nval[c]);
                    __stcg(Dg + c, make_double2(v.ngrad[c * 2], v.ngrad[c * 2 + 1]));
                    __stcg(Dl + c, make_double2(v.nlap[c * 2], v.nlap[c * 2 + 1]));
                }
                const double upd = bs[1] + 1.0;
                const double old_log = bs[0];
                // the reference's triggers; the routine refresh after 64 updates
                // (no other trigger, N <= 24) is the update followed by one
                // Newton-Schulz step on the tensor cores instead of Gauss-Jordan
                const bool trigger = !isfinite(R) || fabs(R) < 1e-5 || bs[2] > 1e8 ||
                                     fabs(R) <= 1e4 * kEps * acc[1];
                const bool refresh = !trigger && upd >= 64.0 && N <= 24;
                bool rebuild = trigger || (upd >= 64.0 && !refresh);
                __syncwarp();
                if (lane == 0) {
                    bs[1] = upd;
                    rabs[jrow] = acc[15];
                }
                // rank-one update (or, on a trigger, the rebuild) and the
                // condition estimate ||D||∞ ||A||∞ of the committed inverse;
                // a rebuild taken for the estimate keeps the estimate from
                // before it, as the reference does.  One call site of the
                // out-of-line Gauss-Jordan.
                double rs_max = 0.0, rd_max = 0.0;
                if (!rebuild) {
#pragma unroll 1
                    for (int a = lane; a < N; a += 32) {
                        const double ca = v.col[a];
                        double ra = 0.0, rb = 0.0;
                        int c = 0;
#pragma unroll 2
                        for (; c + 1 < N; c += 2) {
                            const double x0 = A[a * N + c] - ca * v.rowp[c];
                            const double x1 = A[a * N + c + 1] - ca * v.rowp[c + 1];
                            A[a * N + c] = x0;
                            A[a * N + c + 1] = x1;
                            ra += fabs(x0);
                            rb += fabs(x1);
                        }
                        if (c < N) {
                            const double x0 = A[a * N + c] - ca * v.rowp[c];
                            A[a * N + c] = x0;
                            ra += fabs(x0);
                        }
                        rs_max = fmax(rs_max, ra + rb);
                    }
                }
                __syncwarp();
                for (int a = lane; a < N; a += 32) rd_max = fmax(rd_max, rabs[a]);
                rd_max = warp_max(rd_max);
                double cond = rebuild ? 0.0 : rd_max * warp_max(rs_max);
                bool cond_rebuild = !rebuild && (!isfinite(cond) || cond > 1e8);
                bool refreshed = false;
                if (refresh && !cond_rebuild) {
                    if (ns_refresh_warp(A, D, N) < 1e-6) refreshed = true;
                    else cond_rebuild = true;   // too far from D⁻¹: recompute by Gauss-Jordan
                }
                if (__builtin_expect(rebuild || cond_rebuild, 0)) {
                    gj_rebuild_warp<S>(A, v.work, v.col, D, N, v.misc);
                    if (rebuild) {
                        for (int a = lane; a < N; a += 32) {
                            double rsum = 0.0;
                            for (int c = 0; c < N; ++c) rsum += fabs(A[a * N + c]);
                            rs_max = fmax(rs_max, rsum);
                        }
                        cond = rd_max * warp_max(rs_max);
                    }
                    rebuild = true;
                }
                // (the moved particle's determinant derivatives are not kept:
                // a drift move refreshes them first, the local energy refreshes all)
                if (lane == 0) {
                    bs[2] = cond;
                    if (rebuild) {
                        bs[0] = v.misc[M_LOGDET];
                        bs[1] = 0.0;
                        if (v.misc[M_ERR] != 0.0) v.scal[S_ERR] = 1.0;
                    } else {
                        bs[0] = old_log + log(fabs(R));
                        if (refreshed) bs[1] = 0.0;
                    }
                    v.scal[S_LOGPSI] += bs[0] - old_log;
                }
            }
            double wx = nx, wy = ny;
            wrap2(s, wx, wy);
            if (C && b >= 0 && (wx != nx || wy != ny)) {
                // wrapping moved p by a lattice vector Δ, and every twisted
                // orbital by the same phase e^{iq·Δ}: A's column of p is
                // re-gauged by e^{-iq·Δ} to stay the inverse at the stored positions
                const DevBlock& B = s.blocks[b];
                const int N = B.n, jrow = p - B.first;
                double* Ar = v.scal - s.o_scal + B.oA;
                double* Ai = Ar + ((N * N + 3) & ~3);
                double sa, ca;
                sincos(fma(B.k[1], wy - ny, B.k[0] * (wx - nx)), &sa, &ca);
                for (int m = lane; m < N; m += 32) {
                    const double ar = Ar[m * N + jrow], ai = Ai[m * N + jrow];
                    Ar[m * N + jrow] = ar * ca + ai * sa;
                    Ai[m * N + jrow] = ai * ca - ar * sa;
                }
            }
            if (lane == 0) {
                v.jg[p * 2 + 0] = acc[7];
                v.jg[p * 2 + 1] = acc[8];
                v.jl[p * 2 + 0] = acc[9];
                v.jl[p * 2 + 1] = acc[10];
                v.pos[p * 2 + 0] = wx;
                v.pos[p * 2 + 1] = wy;
                v.scal[S_LOGPSI] += logr - logdr;
            }
            __syncwarp();
        }
        if (dmc || sub == prm.n_sub - 1) {
            __syncwarp();
            const double el = local_energy_warp<S>(s, sm, rec, pairs, npair);
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
    store_fast(s, rec, sm);
}

template <int S, bool ZE, bool C>
__global__ void __launch_bounds__(32, 12) sweep_fast_kernel(const __grid_constant__ DevSys s, double* records,
                                                        int nw, const double* randoms, long stride,
                                                        SweepParams prm, const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    sweep_fast_walker<S, ZE, C>(s, records, w, randoms, stride, prm, pairs, npair, sm);
}

// Packed one-warp sweeps of several contexts (BatchJob, alea_kernels.h),
// all real (C = false) or all complex.
template <bool ZE, bool C>
__global__ void __launch_bounds__(32, 12) sweep_fast_batch_kernel(const BatchJob* __restrict__ jobs, int n_jobs,
                                                              int total, int* next) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int slot;
    for (bool first = true;; first = false) {
        const int w = batch_next(total, next, &slot, first);
        if (w < 0) return;
        const BatchJob& J = jobs[batch_job_of(jobs, n_jobs, w)];
        sweep_fast_walker<2, ZE, C>(*J.sys, J.records, w - J.first, J.randoms, J.stride, J.prm, J.pairs, J.npair,
                                    sm);
    }
}

cudaError_t launch_sweep_fast_batch(bool zero_energy, bool complex_det, const BatchJob* jobs, int n_jobs, int total,
                                    int grid, size_t smem, int* next, cudaStream_t st) {
    if (complex_det)
        sweep_fast_batch_kernel<false, true><<<grid, 32, smem, st>>>(jobs, n_jobs, total, next);
    else if (zero_energy)
        sweep_fast_batch_kernel<true, false><<<grid, 32, smem, st>>>(jobs, n_jobs, total, next);
    else
        sweep_fast_batch_kernel<false, false><<<grid, 32, smem, st>>>(jobs, n_jobs, total, next);
    return cudaGetLastError();
}

int fast_batch_ctas_per_sm(bool complex_det, size_t smem) {
    int n = 0;
    const cudaError_t e =
        complex_det ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_fast_batch_kernel<false, true>, 32, smem)
                    : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_fast_batch_kernel<false, false>, 32,
                                                                    smem);
    return e == cudaSuccess ? std::max(n, 1) : 1;
}

// Does the system have a zero-energy pair term (the out-of-line radial form)?
static bool has_zero_energy(const DevSys& s) {
    for (int t = 0; t < s.nterms; ++t)
        if (s.terms[t].kind == 2) return true;
    return false;
}

// Complex determinants take the one-warp sweep without zero-energy pair
// terms (no such system is built; the form is not compiled).
bool fast_sweep_eligible(const DevSys& s) {
    return s.dim == 2 && s.nbf == 0 && s.pair_by_group && s.np <= 64 && s.maxN <= 64 && s.nkJ <= 64 &&
           s.ngroups <= 8 && !(s.cplx && has_zero_energy(s));
}

cudaError_t reserve_smem_fast(size_t smem) {
    for (const void* k : {reinterpret_cast<const void*>(sweep_fast_kernel<2, false, false>),
                          reinterpret_cast<const void*>(sweep_fast_kernel<2, true, false>),
                          reinterpret_cast<const void*>(sweep_fast_kernel<2, false, true>),
                          reinterpret_cast<const void*>(sweep_fast_batch_kernel<false, false>),
                          reinterpret_cast<const void*>(sweep_fast_batch_kernel<true, false>),
                          reinterpret_cast<const void*>(sweep_fast_batch_kernel<false, true>)}) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_sweep_fast(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records,
                              const double* randoms, long stride, const SweepParams& prm, const int2* pairs,
                              int npair) {
    (void)smem;
    const size_t bytes = static_cast<size_t>(s.f_total) * 8;
    if (s.cplx)
        sweep_fast_kernel<2, false, true><<<nw, 32, bytes, st>>>(s, records, nw, randoms, stride, prm, pairs, npair);
    else if (has_zero_energy(s))
        sweep_fast_kernel<2, true, false><<<nw, 32, bytes, st>>>(s, records, nw, randoms, stride, prm, pairs, npair);
    else
        sweep_fast_kernel<2, false, false><<<nw, 32, bytes, st>>>(s, records, nw, randoms, stride, prm, pairs,
                                                                  npair);
    return cudaGetLastError();
}

}  // namespace alea_gpu
