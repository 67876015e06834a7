// The one-warp sweep (sm_100a) for Jastrow-only systems of up to 256
// particles: no determinant, pair Jastrows by group at the minimum image, no
// image sums (the dipolar bosons of the serving mix).  One CTA of 32 threads
// per walker, the walker's state in the one-warp shared-memory layout of
// alea_fast.cu.
//
// Algorithms restated from the reference (ItaloAlb/alea), in the steps of
// the generic sweep of alea_kernels.cu:
//   sweep          src/qmc/vmc.cpp:82-155, src/qmc/dmc.cpp:203-337,
//                  src/numerics/green_function.h:20-58
//   pair Jastrows  src/wavefunction/pade_jastrow.cpp:347-634,
//                  src/wavefunction/zero_energy_jastrow.h:16-55
//   E_L, weights   src/hamiltonian/kinetic.cpp:45-72,
//                  src/hamiltonian/inverse_power.h:11-62,
//                  src/qmc/population_control.cpp:56-77
//
// Work split.  Lane l owns partners l + 32j; a move walks them two slots at
// a time (64 partners per pass, both slots' radial evaluations in flight
// together), keeps each partner's derivative change in `work` for the
// commit, and meets the move's five sums (log J, p's new gradient and
// Laplacian) in one warp all-reduce, so every lane takes the accept decision
// itself.  The next particle's three random numbers are loaded while the
// current move runs.  The generic CTA sweep synchronises the block several
// times a move; here a move has no block barrier.
#include "alea_warp.cuh"

namespace alea_gpu {

namespace {

constexpr int kBosonSlots = 8;   // 256 partners per lane slot set

template <bool ZE>
__device__ __forceinline__ void sweep_boson_walker(const DevSys& s, double* records, int w, const double* randoms,
                                                   long stride, const SweepParams& prm, const int2* pairs,
                                                   int npair, double* sm) {
    const int lane = threadIdx.x;
    double* rec = records + static_cast<long>(w) * s.rec;
    load_fast(s, rec, sm);
    const Smem v = view_fast(s, sm, false);
    const int np = s.np;
    const bool dmc = prm.mode == 1;
    const bool drift = dmc || prm.drift != 0;
    double zrm = 0.0;   // largest matching radius of the zero-energy terms
    if constexpr (ZE)
        for (int t = 0; t < s.nterms; ++t)
            if (s.terms[t].kind == 2) zrm = fmax(zrm, s.terms[t].ze_rm);
    // an idle slot runs its radial terms at this distance and contributes nothing
    const double idle_r = fmax(1.0, 2.0 * zrm);
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
        double r0n = __ldcs(rnd + w), r1n = __ldcs(rnd + stride + w), un = __ldcs(rnd + 2 * stride + w);
        for (int p = 0; p < np; ++p) {
            const double r0 = r0n, r1 = r1n, u = un;
            if (p + 1 < np) {
                const double* g = rnd + static_cast<long>(p + 1) * 3 * stride + w;
                r0n = __ldcs(g);
                r1n = __ldcs(g + stride);
                un = __ldcs(g + 2 * stride);
            }
            const int gp = __ldg(s.group_of + p);
            const double px = v.pos[p * 2], py = v.pos[p * 2 + 1];
            // ── proposal (every lane, identical arithmetic) ──
            const double im0 = ldg_keep(s.inv_mass + p * 2), im1 = ldg_keep(s.inv_mass + p * 2 + 1);
            const double tm = prm.tau * im0;
            const double gx = v.jg[p * 2], gy = v.jg[p * 2 + 1];
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
            // ── pair terms: log J, p's new ∇ and ∂², each partner's change ──
            // acc: 0 log J, 1-2 ∇, 3-4 ∂² (5-7 unused)
            double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 1
            for (int k0 = lane; k0 < np; k0 += 64) {
                unsigned cm[2];
                double rn[2], ro[2], dnx[2], dny[2], dox[2], doy[2];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int k = k0 + 32 * j;
                    cm[j] = (k < np && k != p) ? static_cast<unsigned>(s.gterms[gp][__ldg(s.group_of + k)]) : 0u;
                    const double kx0 = cm[j] ? v.pos[k * 2] : px + 1.0;
                    const double ky0 = cm[j] ? v.pos[k * 2 + 1] : py;
                    rn[j] = fold2(s, nx, ny, kx0, ky0, dnx[j], dny[j]);
                    ro[j] = fold2(s, px, py, kx0, ky0, dox[j], doy[j]);
                    if (!cm[j]) rn[j] = ro[j] = idle_r;
                }
                double uo[2], duo[2], d2uo[2], un2[2], dun[2], d2un[2];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const DevTerm& T = s.terms[cm[j] ? __ffs(cm[j]) - 1 : 0];
                    radial_w<ZE>(T, ro[j], uo[j], duo[j], d2uo[j]);
                    radial_w<ZE>(T, rn[j], un2[j], dun[j], d2un[j]);
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    for (unsigned bits = cm[j] & (cm[j] - 1); bits; bits &= bits - 1) {
                        const DevTerm& T = s.terms[__ffs(bits) - 1];
                        double a0, a1, a2, b0, b1, b2;
                        radial_w<ZE>(T, ro[j], a0, a1, a2);
                        radial_w<ZE>(T, rn[j], b0, b1, b2);
                        uo[j] += a0;
                        duo[j] += a1;
                        d2uo[j] += a2;
                        un2[j] += b0;
                        dun[j] += b1;
                        d2un[j] += b2;
                    }
                }
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    if (!cm[j]) continue;
                    const double irn = 1.0 / rn[j], iro = 1.0 / ro[j];
                    acc[0] += un2[j] - uo[j];
                    double* dj = v.work + (k0 + 32 * j) * 4;
                    {
                        const double dor = dnx[j] * irn;
                        acc[1] += dun[j] * dor;
                        acc[3] += d2un[j] * dor * dor + dun[j] * irn * (1.0 - dor * dor);
                        const double dor_old = -dox[j] * iro, dor_new = -dnx[j] * irn;
                        dj[0] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[2] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0 - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0 - dor_old * dor_old));
                    }
                    {
                        const double dor = dny[j] * irn;
                        acc[2] += dun[j] * dor;
                        acc[4] += d2un[j] * dor * dor + dun[j] * irn * (1.0 - dor * dor);
                        const double dor_old = -doy[j] * iro, dor_new = -dny[j] * irn;
                        dj[1] = dun[j] * dor_new - duo[j] * dor_old;
                        dj[3] = (d2un[j] * dor_new * dor_new + dun[j] * irn * (1.0 - dor_new * dor_new)) -
                                (d2uo[j] * dor_old * dor_old + duo[j] * iro * (1.0 - dor_old * dor_old));
                    }
                }
            }
            warp_allsum<8>(acc);
            const double logr = acc[0];
            // ── accept / reject (every lane, identical decision) ──
            const double ngx_t = acc[1], ngy_t = acc[2];
            const double dx = nx - px, dy = ny - py;
            const double tm0 = prm.tau * im0, tm1 = prm.tau * im1;
            bool accept;
            if (dmc) {
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
            // ── commit: partners' changes, p's new derivatives and position ──
            if (lane == 0) v.scal[S_NACC] += 1.0;
#pragma unroll 1
            for (int k = lane; k < np; k += 32) {
                if (k == p || s.gterms[gp][__ldg(s.group_of + k)] == 0) continue;
                const double* dj = v.work + k * 4;
                v.jg[k * 2 + 0] += dj[0];
                v.jg[k * 2 + 1] += dj[1];
                v.jl[k * 2 + 0] += dj[2];
                v.jl[k * 2 + 1] += dj[3];
            }
            if (lane == 0) {
                v.jg[p * 2 + 0] = acc[1];
                v.jg[p * 2 + 1] = acc[2];
                v.jl[p * 2 + 0] = acc[3];
                v.jl[p * 2 + 1] = acc[4];
                double wx = nx, wy = ny;
                wrap2(s, wx, wy);
                v.pos[p * 2 + 0] = wx;
                v.pos[p * 2 + 1] = wy;
                v.scal[S_LOGPSI] += logr;
            }
            __syncwarp();
        }
        if (dmc || sub == prm.n_sub - 1) {
            __syncwarp();
            const double el = local_energy_warp<kBosonSlots>(s, sm, rec, pairs, npair);
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

template <bool ZE>
__global__ void __launch_bounds__(32, 8) sweep_boson_kernel(const __grid_constant__ DevSys s, double* records,
                                                            int nw, const double* randoms, long stride,
                                                            SweepParams prm, const int2* pairs, int npair) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    sweep_boson_walker<ZE>(s, records, w, randoms, stride, prm, pairs, npair, sm);
}

// Packed one-warp Jastrow-only sweeps of several contexts (BatchJob).
template <bool ZE>
__global__ void __launch_bounds__(32, 8) sweep_boson_batch_kernel(const BatchJob* __restrict__ jobs, int n_jobs,
                                                                  int total, int* next) {
    extern __shared__ __align__(16) double sm[];
    __shared__ int slot;
    for (bool first = true;; first = false) {
        const int w = batch_next(total, next, &slot, first);
        if (w < 0) return;
        const BatchJob& J = jobs[batch_job_of(jobs, n_jobs, w)];
        sweep_boson_walker<ZE>(*J.sys, J.records, w - J.first, J.randoms, J.stride, J.prm, J.pairs, J.npair, sm);
    }
}

bool has_zero_energy_b(const DevSys& s) {
    for (int t = 0; t < s.nterms; ++t)
        if (s.terms[t].kind == 2) return true;
    return false;
}

}  // namespace

bool boson_sweep_eligible(const DevSys& s) {
    return s.dim == 2 && s.nblocks == 0 && s.nbf == 0 && s.nkJ == 0 && s.pair_by_group && s.np > 64 &&
           s.np <= 32 * kBosonSlots && s.ngroups <= 8;
}

cudaError_t reserve_smem_boson(size_t smem) {
    for (const void* k : {reinterpret_cast<const void*>(sweep_boson_kernel<false>),
                          reinterpret_cast<const void*>(sweep_boson_kernel<true>),
                          reinterpret_cast<const void*>(sweep_boson_batch_kernel<false>),
                          reinterpret_cast<const void*>(sweep_boson_batch_kernel<true>)}) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_sweep_boson(int nw, cudaStream_t st, const DevSys& s, double* records, const double* randoms,
                               long stride, const SweepParams& prm, const int2* pairs, int npair) {
    const size_t bytes = static_cast<size_t>(s.f_total) * 8;
    if (has_zero_energy_b(s))
        sweep_boson_kernel<true><<<nw, 32, bytes, st>>>(s, records, nw, randoms, stride, prm, pairs, npair);
    else
        sweep_boson_kernel<false><<<nw, 32, bytes, st>>>(s, records, nw, randoms, stride, prm, pairs, npair);
    return cudaGetLastError();
}

cudaError_t launch_sweep_boson_batch(bool zero_energy, const BatchJob* jobs, int n_jobs, int total, int grid,
                                     size_t smem, int* next, cudaStream_t st) {
    if (zero_energy)
        sweep_boson_batch_kernel<true><<<grid, 32, smem, st>>>(jobs, n_jobs, total, next);
    else
        sweep_boson_batch_kernel<false><<<grid, 32, smem, st>>>(jobs, n_jobs, total, next);
    return cudaGetLastError();
}

int boson_batch_ctas_per_sm(size_t smem) {
    int n = 0;
    const cudaError_t e =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sweep_boson_batch_kernel<true>, 32, smem);
    return e == cudaSuccess ? std::max(n, 1) : 1;
}

}  // namespace alea_gpu
