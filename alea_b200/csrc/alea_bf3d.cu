// Walker kernels in three dimensions (sm_100a): the backflow electron gas
// and, with no backflow channels, plain determinants of 3-D orbitals.
//
// Restated from the reference (ItaloAlb/alea), whose backflow determinant,
// Jastrows, kinetic energy and drivers are dimension-generic:
//   backflow       src/wavefunction/backflow_slater_determinant.cpp:28-65
//                  (invert), :520-579 (ratio_batch), :600-697 (commit,
//                  refresh_walker, all_derivatives), backflow_transformation.cpp
//                  :120-284 (shift, particle tables, Jacobian columns),
//                  backflow_function.h:11-42 (η)
//   orbitals       src/wavefunction/orbital_set.h:185-224 (Gaussians),
//                  :436-474 (plane waves; the reference builds no 3-D shells,
//                  the caller passes the k-vectors)
//   pair Jastrows  src/wavefunction/radial_pair_jastrow_impl.h (Drummond,
//                  minimum-image Padé)
//   E_L            src/hamiltonian/kinetic.cpp:45-72; the 3-D Ewald sum is
//                  this project's own (the reference refuses 3-D Ewald,
//                  src/numerics/ewald_breakup.cpp:211-213): Σ_{i<j} q_i q_j
//                  [ε⁻¹/r − f_l(r)] (r < r_c) + Σ_k w_k |ρ(k)|² + constants
//   sweep          src/qmc/vmc.cpp:82-155, src/qmc/dmc.cpp:203-337,
//                  src/numerics/green_function.h:20-58
//
// One CTA of 128 threads per walker.  A move of particle p changes every
// quasi-coordinate that p displaces, so each determinant p touches is formed
// anew and inverted by pivoted Gauss-Jordan (its ratio is det M'/det M, no
// rank-one update applies), one warp per determinant so that the two spins'
// determinants invert at once; the inverse A', F' = A'ᵀ∇φ(x') and
// log|det M'| are kept pending and committed on acceptance.  The moves run
// in their own launch (sweep3_kernel, the moves' smaller shared-memory
// layout); the refresh that follows (refresh3_kernel) rebuilds x from the
// positions and every particle's ∇ and per-dimension ∂² ln|D| from the
// committed A and F: T = Aᵀ∂∂φ, G^a = Aᵀ∂_aφ (three N×N×N products on the
// FP64 tensor cores) and the Jacobian columns ∂x_t/∂r_k^β (ln|D|'s
// Laplacian is Σ F·∂²x + Σ v v T − tr((G·v)²)), then the local energy.
//
// Record of a 3-D walker (doubles): positions, Jastrow ∇/∂², two zero planes
// (the k-space planes of the 2-D layout, read by the download), determinant
// ∇/∂², the scalars, then per determinant x (3N), A (N²), F (3N) and
// (log|det|, sign).  All of it is hot: each launch stages it in shared
// memory, in and out as one bulk copy each.
#include "alea_warp.cuh"

namespace alea_gpu {

namespace {

constexpr int kNT3 = 128;

// misc slots of the 3-D kernels
enum : int {
    T_LOGR = 0, T_SIGN, T_ACC, T_ERR, T_U, T_SCF, T_GO /* 3 */ = 6, T_GN /* 3 */ = 9, T_LS /* 3 */ = 12,
    T_BAD = 15, T_JG /* 3: p's new Jastrow gradient */ = 16, T_JL /* 3: and Laplacian */ = 19
};

struct V3 {
    double *pos, *jg, *jl, *kg, *kl, *sg, *sl, *scal;
    double *newpos, *misc, *red, *col, *work, *mwork;
};

__device__ __forceinline__ V3 view3(const DevSys& s, double* sm) {
    V3 v;
    v.pos = sm + s.o_pos;
    v.jg = sm + s.o_jg;
    v.jl = sm + s.o_jl;
    v.kg = sm + s.o_kg;
    v.kl = sm + s.o_kl;
    v.sg = sm + s.o_sg;
    v.sl = sm + s.o_sl;
    v.scal = sm + s.o_scal;
    v.newpos = sm + s.t_newpos;
    v.misc = sm + s.t_misc;
    v.red = sm + s.t_red;
    v.col = sm + s.t_col;
    v.work = sm + s.t_work;
    v.mwork = sm + s.t_mwork;
    return v;
}

// Minimum-image displacement a - b (orthorhombic fold, or none in an open
// cell) and its length.
__device__ __forceinline__ double dist3(const DevSys& s, const double* a, const double* b, double* del) {
    del[0] = a[0] - b[0];
    del[1] = a[1] - b[1];
    del[2] = a[2] - b[2];
    min_image(s, del);
    return sqrt(fma(del[2], del[2], fma(del[1], del[1], del[0] * del[0])));
}

// One backflow pair r_ij = ri - rj: adds sign·η r_ij to x; fills B[a][b] =
// ∂(η r_a)/∂r_b and S[a][b] = ∂²(η r_a)/∂r_b² (3x3, row a) when B is given.
// False beyond the cutoff.
__device__ __forceinline__ bool bf3_pair(const DevSys& s, const DevBFCh& C, const double* ri, const double* rj,
                                         double sign, double* x, double* B, double* S) {
    double del[3];
    const double r = dist3(s, ri, rj, del);
    if (r >= C.L) return false;
    double eta, e1, e2;
    bf_eta(C, r, eta, e1, e2);
    x[0] += sign * eta * del[0];
    x[1] += sign * eta * del[1];
    x[2] += sign * eta * del[2];
    if (B) {
        const double inv_r = r > 0.0 ? 1.0 / r : 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                B[a * 3 + b] = (a == b ? eta : 0.0) + e1 * del[a] * del[b] * inv_r;
                if (S) {
                    const double rb2 = del[b] * del[b] * inv_r * inv_r;
                    S[a * 3 + b] = (a == b ? 2.0 * e1 * del[b] * inv_r : 0.0) +
                                   del[a] * (e2 * rb2 + e1 * inv_r * (1.0 - rb2));
                }
            }
    }
    return true;
}

// Orbital m at x: value and gradient.
__device__ __forceinline__ void bf3_orbital(const DevSys& s, const DevBF& D, int m, const double* x, double& val,
                                            double* g) {
    if (D.type == 0) {
        const double* k = D.k + m * 3;
        double sn, c;
        sincos(fma(k[2], x[2], fma(k[1], x[1], k[0] * x[0])), &sn, &c);
        const bool is_s = D.is_sin[m] != 0.0;
        const double v = is_s ? sn : c, dv = is_s ? c : -sn;
        val = v;
        g[0] = k[0] * dv;
        g[1] = k[1] * dv;
        g[2] = k[2] * dv;
    } else {
        const double al = D.alphas[m];
        double del[3];
        const double r = dist3(s, x, D.centers + m * 3, del);
        const double phi = exp(-al * r * r);
        val = phi;
        g[0] = -2.0 * al * del[0] * phi;
        g[1] = -2.0 * al * del[1] * phi;
        g[2] = -2.0 * al * del[2] * phi;
    }
}

// ∂_a∂_b φ_m at x (val: φ_m(x)).
__device__ __forceinline__ double bf3_hess(const DevSys& s, const DevBF& D, int m, const double* x, double val,
                                           int a, int b) {
    if (D.type == 0) return -D.k[m * 3 + a] * D.k[m * 3 + b] * val;
    const double al = D.alphas[m];
    double del[3];
    dist3(s, x, D.centers + m * 3, del);
    return (4.0 * al * al * del[a] * del[b] - (a == b ? 2.0 * al : 0.0)) * val;
}

__device__ __forceinline__ bool in_sources(const DevBFCh& C, int k) { return k >= C.sf && k < C.sl; }

// Plane-wave orbitals m and m + 1 are the cosine and the sine of one k.
__device__ __forceinline__ bool pw_pair(const DevBF& D, int m) {
    if (m < 0 || m + 1 >= D.n || D.is_sin[m] != 0.0 || D.is_sin[m + 1] == 0.0) return false;
    const double* k = D.k + m * 3;
    return k[0] == k[3] && k[1] == k[4] && k[2] == k[5];
}

// The orbital units of a determinant, for a move's new matrices: units[d][u]
// is the orbital index of unit u (with kUnitPair: it and the next orbital
// are a plane wave's cosine and sine), units[d][32] the number of units.
// Built by the first warp; the caller's barrier publishes it.
constexpr unsigned char kUnitPair = 0x40;

__device__ void build_units(const DevSys& s, unsigned char (*units)[33]) {
    if (threadIdx.x >= 32) return;
    const int m = threadIdx.x;
    for (int d = 0; d < s.nbf; ++d) {
        const DevBF& D = s.bf[d];
        const bool pw = D.type == 0;
        const bool first = m < D.n && !(pw && pw_pair(D, m - 1));
        const unsigned mask = __ballot_sync(0xffffffffu, first);
        if (first)
            units[d][__popc(mask & ((1u << m) - 1u))] =
                static_cast<unsigned char>(m | (pw && pw_pair(D, m) ? kUnitPair : 0));
        if (m == 0) units[d][32] = static_cast<unsigned char>(__popc(mask));
    }
}

// Rows r0 .. r0 + B - 1 of A lose their multiple mult[r] of the pivot row's
// entry pk in this lane's column: B rows' loads in flight, then their
// updates, the multipliers as 16-byte loads (mult + r0 16-byte aligned).
template <int B>
__device__ __forceinline__ void gj_rows(double* A, const double* mult, int N, int r0, int lane, double pk) {
    double f[B], y[B];
    const double2* m2 = reinterpret_cast<const double2*>(mult + r0);
#pragma unroll
    for (int u = 0; u < B / 2; ++u) {
        const double2 q = m2[u];
        f[2 * u] = q.x;
        f[2 * u + 1] = q.y;
    }
#pragma unroll
    for (int u = 0; u < B; ++u) y[u] = A[(r0 + u) * N + lane];
#pragma unroll
    for (int u = 0; u < B; ++u) A[(r0 + u) * N + lane] = fma(-f[u], pk, y[u]);
}

// In-place pivoted Gauss-Jordan of the N×N matrix A (N <= 32, row-major in
// shared memory) by the calling warp: A becomes A⁻¹; out[0] = log|det A|,
// out[1] = its sign, out[2] = 1 when every pivot is finite and nonzero.
// Lane c owns column c.  The pivot of column k is the first row of largest
// |x| at or below k (the rule of the reference's invert,
// backflow_slater_determinant.cpp:28-65), found by integer max/min warp
// reductions on the bits of |x| (order-preserving for non-negative doubles;
// a NaN never wins); row k is scaled by 1/pivot, the other rows lose their
// multiple of it (multipliers in `mult`), and the row exchanges (`perm`) are
// undone as column exchanges at the end.  The exchange, the scaling and the
// multipliers of a pivot share one phase (they touch disjoint entries), and
// log|det| is one log per lane at the end.  No block barrier: two warps
// invert two determinants at once.  (A register-resident form, a column per
// lane with the multipliers broadcast by shuffles, ran 2.3x slower here.)
__device__ void gj_warp_signed(double* A, int N, double* mult, int* perm, double* out) {
    const unsigned all = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    __syncwarp();
    double sign = 1.0, my_pivot = 1.0;   // lane k keeps pivot k: one log per lane at the end
    bool bad = false;
    const bool vec = (reinterpret_cast<uintptr_t>(mult) & 15u) == 0;
    for (int k = 0; k < N; ++k) {
        const double x = lane < N ? A[lane * N + k] : 0.0;   // column k, row = lane
        unsigned long long key = 0ull;
        if (lane >= k && lane < N)
            key = isnan(x) ? 0ull : static_cast<unsigned long long>(__double_as_longlong(fabs(x))) + 1ull;
        const unsigned hi = static_cast<unsigned>(key >> 32), lo = static_cast<unsigned>(key);
        const unsigned mhi = __reduce_max_sync(all, hi);
        const unsigned mlo = __reduce_max_sync(all, hi == mhi ? lo : 0u);
        const bool cand = key != 0ull && hi == mhi && lo == mlo;
        const unsigned prow = __reduce_min_sync(all, cand ? static_cast<unsigned>(lane) : 0xffffffffu);
        const bool none = mhi == 0u && mlo == 0u;
        const int piv = none ? k : static_cast<int>(prow);
        double diag = __shfl_sync(all, x, piv);
        const double xkk = __shfl_sync(all, x, k);
        if (none) diag = 0.0;
        bad |= diag == 0.0 || !isfinite(diag);
        if (lane == k) my_pivot = diag;
        if (diag < 0.0) sign = -sign;
        if (piv != k) sign = -sign;
        const double inv = __drcp_rn(diag);
        double pk = 0.0;
        if (lane < N) {
            // rows k and piv exchanged and row k scaled (lane = column; column k's
            // other entries are the multipliers' business below) ...
            const double xk = A[k * N + lane], xp = A[piv * N + lane];
            if (piv != k && lane != k) A[piv * N + lane] = xk;
            pk = (lane == k ? 1.0 : (piv != k ? xp : xk)) * inv;
            A[k * N + lane] = pk;
            // ... and, lane = row, the multipliers: column k after the exchange,
            // which then starts from 0 (no entry of another phase's)
            const double m = lane == k ? 0.0 : (lane == piv ? xkk : x);
            mult[lane] = m;
            if (lane != k) A[lane * N + k] = 0.0;
        }
        if (lane == 0) perm[k] = piv;
        __syncwarp();
        if (lane < N) {
            if (vec) {   // whole blocks of 8, then 4, 2 and 1 rows, multipliers in 16-byte loads
                int r0 = 0;
                for (; r0 + 8 <= N; r0 += 8) gj_rows<8>(A, mult, N, r0, lane, pk);
                if (r0 + 4 <= N) {
                    gj_rows<4>(A, mult, N, r0, lane, pk);
                    r0 += 4;
                }
                if (r0 + 2 <= N) {
                    gj_rows<2>(A, mult, N, r0, lane, pk);
                    r0 += 2;
                }
                if (r0 < N) A[r0 * N + lane] = fma(-mult[r0], pk, A[r0 * N + lane]);
            } else {
                for (int r0 = 0; r0 < N; r0 += 8) {   // eight rows' loads in flight, then their updates
                    double f[8], y[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const bool on = r0 + u < N;
                        f[u] = on ? mult[r0 + u] : 0.0;
                        y[u] = on ? A[(r0 + u) * N + lane] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (r0 + u < N) A[(r0 + u) * N + lane] = fma(-f[u], pk, y[u]);
                }
            }
        }
        __syncwarp();
    }
    for (int k = N - 1; k >= 0; --k) {
        const int pk = perm[k];
        if (pk != k && lane < N) {
            const double t = A[lane * N + k];
            A[lane * N + k] = A[lane * N + pk];
            A[lane * N + pk] = t;
        }
        __syncwarp();
    }
    const double logdet = warp_sum(lane < N ? log(fabs(my_pivot)) : 0.0);
    if (lane == 0) {
        out[0] = logdet;
        out[1] = sign;
        out[2] = bad ? 0.0 : 1.0;
    }
    __syncwarp();
}

// ∂_k ln|D| = F_k (1 + Σ_j B(r_kj)) - Σ_t F_t B(r_tk) at the positions (with
// `moved` at npos), summed over the CTA; every thread returns it.
template <int NT>
__device__ void bf3_grad(const DevSys& s, const DevBF& D, const double* F, const double* pos, int k, int moved,
                         const double* npos, double* red, double* g) {
    const int N = D.n, np = s.np;
    const double* rk = k == moved ? npos : pos + k * 3;
    const int tk = (k >= D.first && k < D.last) ? k - D.first : -1;
    double acc[3] = {0.0, 0.0, 0.0};
    if (tk >= 0) {
        const double* Fk = F + tk * 3;
        if (threadIdx.x == 0) {
            acc[0] += Fk[0];
            acc[1] += Fk[1];
            acc[2] += Fk[2];
        }
        for (int j = threadIdx.x; j < np; j += NT) {
            if (j == k) continue;
            const double* rj = j == moved ? npos : pos + j * 3;
            for (int c = 0; c < D.nch; ++c) {
                if (!in_sources(D.ch[c], j)) continue;
                double unused[3] = {0, 0, 0}, B[9];
                if (!bf3_pair(s, D.ch[c], rk, rj, 1.0, unused, B, nullptr)) continue;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int b = 0; b < 3; ++b) acc[b] += Fk[a] * B[a * 3 + b];
            }
        }
    }
    for (int t = threadIdx.x; t < N; t += NT) {
        const int P = D.first + t;
        if (P == k) continue;
        const double* rt = P == moved ? npos : pos + P * 3;
        for (int c = 0; c < D.nch; ++c) {
            if (!in_sources(D.ch[c], k)) continue;
            double unused[3] = {0, 0, 0}, B[9];
            if (!bf3_pair(s, D.ch[c], rt, rk, 1.0, unused, B, nullptr)) continue;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) acc[b] -= F[t * 3 + a] * B[a * 3 + b];
        }
    }
    block_sum<NT>(acc, red);
    g[0] = acc[0];
    g[1] = acc[1];
    g[2] = acc[2];
}

// ───────────────────────── pair Jastrows ────────────────────────────────

// Does pair range q of term T couple i with j (i != j)?
__device__ __forceinline__ bool term_couples(const DevTerm& T, int q, int i, int j) {
    const int af = T.pairs[q][0], al = T.pairs[q][1], bf = T.pairs[q][2], bl = T.pairs[q][3];
    const bool ia = i >= af && i < al, ib = i >= bf && i < bl;
    const bool ja = j >= af && j < al, jb = j >= bf && j < bl;
    return (ia && jb) || (ib && ja);
}

__device__ __forceinline__ bool any_term_couples(const DevTerm& T, int i, int j) {
    for (int q = 0; q < T.npairs; ++q)
        if (term_couples(T, q, i, j)) return true;
    return false;
}

// Every particle's Jastrow ∇ and per-dimension ∂² (jg, jl) and ln J.
template <int NT>
__device__ double jastrow_all(const DevSys& s, const V3& v) {
    const int np = s.np;
    double lj = 0.0;
    for (int i = threadIdx.x; i < np; i += NT) {
        double g[3] = {0, 0, 0}, l[3] = {0, 0, 0};
        for (int t = 0; t < s.nterms; ++t) {
            const DevTerm& T = s.terms[t];
            for (int j = 0; j < np; ++j) {
                if (j == i || !any_term_couples(T, i, j)) continue;
                double del[3];
                const double r = dist3(s, v.pos + i * 3, v.pos + j * 3, del);
                double u, du, d2u;
                radial(T, r, u, du, d2u);
                if (j > i) lj += u;
                const double ir = 1.0 / r;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double dor = del[d] * ir;
                    g[d] += du * dor;
                    l[d] += d2u * dor * dor + du * ir * (1.0 - dor * dor);
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v.jg[i * 3 + d] = g[d];
            v.jl[i * 3 + d] = l[d];
        }
    }
    double acc[1] = {lj};
    block_sum<NT>(acc, v.red);
    return acc[0];
}

// ───────────────────────── backflow refresh ─────────────────────────────

// Determinant d's x from the positions and every particle's ∇, ∂² ln|D|
// added into sg/sl, from the committed A and F (refresh_walker); with
// `invert`, A, F and (log|det|, sign) are first computed anew by pivoted
// Gauss-Jordan (evaluate_batch).  Work area: M (N²), orbital rows
// [(t·N + m)·4 + (φ, ∂x, ∂y, ∂z)] (4N²), G^a[j][r] (3N²), T (6N), the x
// rebuild's slice sums (12N; 48N for the per-particle warps when N < 12).
template <int NT>
__device__ void bf3_refresh(const DevSys& s, const V3& v, double* sm, int d, bool invert) {
    const DevBF& D = s.bf[d];
    const int N = D.n, np = s.np;
    double* x = sm + D.oX;
    double* A = sm + D.oA;
    double* F = sm + D.oF;
    double* ls = sm + D.oLS;
    double* M = v.work;
    double* R = M + N * N;
    double* G = R + 4 * N * N;
    double* T = G + 3 * N * N;
    double* J = T + 6 * N;
    __syncthreads();
    {   // x from the positions: row t's source sums in 4 slices (one thread per
        // row and slice, partial sums in J's area), then added in slice order
        constexpr int kS = 4;
        for (int e = threadIdx.x; e < N * kS; e += NT) {
            const int t = e / kS, sl = e % kS, P = D.first + t;
            double acc[3] = {0.0, 0.0, 0.0};
            for (int c = 0; c < D.nch; ++c)
                for (int j = D.ch[c].sf + sl; j < D.ch[c].sl; j += kS)
                    if (j != P) bf3_pair(s, D.ch[c], v.pos + P * 3, v.pos + j * 3, 1.0, acc, nullptr, nullptr);
            J[e * 3] = acc[0];
            J[e * 3 + 1] = acc[1];
            J[e * 3 + 2] = acc[2];
        }
        __syncthreads();
        for (int t = threadIdx.x; t < N; t += NT) {
            const double* rp = v.pos + (D.first + t) * 3;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                double sum = 0.0;
#pragma unroll
                for (int sl = 0; sl < kS; ++sl) sum += J[(t * kS + sl) * 3 + a];
                x[t * 3 + a] = rp[a] + sum;
            }
        }
    }
    __syncthreads();
    for_each_elem<NT>(N, [&](int t, int m) {
        double val, g[3];
        bf3_orbital(s, D, m, x + t * 3, val, g);
        double* r = R + (t * N + m) * 4;
        r[0] = val;
        r[1] = g[0];
        r[2] = g[1];
        r[3] = g[2];
        if (invert) M[t * N + m] = val;
    });
    __syncthreads();
    if (invert) {
        bf_invert<NT>(N, M, A, v.col, v.misc + T_LS);
        __syncthreads();
        if (threadIdx.x == 0) {
            if (v.misc[T_LS + 2] == 0.0) v.misc[T_ERR] = 1.0;
            ls[0] = v.misc[T_LS];
            ls[1] = v.misc[T_LS + 1];
        }
        __syncthreads();
        if (v.misc[T_LS + 2] == 0.0) return;
        for (int e = threadIdx.x; e < 3 * N; e += NT) {   // F_t = Σ_m A[m][t] ∇φ_m(x_t)
            const int t = e / 3, a = e % 3;
            double acc = 0.0;
            for (int m = 0; m < N; ++m) acc = fma(A[m * N + t], R[(t * N + m) * 4 + 1 + a], acc);
            F[t * 3 + a] = acc;
        }
    }
    // G^a = Aᵀ (∂_a Φ)ᵀ, G^a[j][r] = Σ_m A[m][j] ∂_a φ_m(x_r): three N×N×N products
    // on the FP64 tensor cores, 8×8 output tiles dealt to the warps, k in
    // slabs of 4 (mma.sync m8n8k4 .f64; lane 4g + t holds P[g][t], Q[t][g]
    // and C[g][2t..2t+1] of a tile, zero-padded beyond N)
    {
        const int lane = threadIdx.x & 31, g = lane >> 2, tq = lane & 3, warp = threadIdx.x >> 5;
        const int nt = (N + 7) >> 3, nk = (N + 3) >> 2;
        for (int job = warp; job < 3 * nt * nt; job += NT / 32) {
            const int a = job / (nt * nt), jt = (job / nt) % nt, rt = job % nt;
            const int j = jt * 8 + g, r = rt * 8 + g;
            double c[2] = {0.0, 0.0};
            for (int kt = 0; kt < nk; ++kt) {
                const int m = kt * 4 + tq;
                const double pa = (j < N && m < N) ? A[m * N + j] : 0.0;
                const double qb = (r < N && m < N) ? R[(r * N + m) * 4 + 1 + a] : 0.0;
                dmma_m8n8k4(c, pa, qb);
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int rc = rt * 8 + 2 * tq + i;
                if (j < N && rc < N) G[a * N * N + j * N + rc] = c[i];
            }
        }
    }
    // T_t^{ab} = Σ_m A[m][t] ∂_a∂_b φ_m(x_t)
    for (int e = threadIdx.x; e < 6 * N; e += NT) {
        const int t = e / 6, q = e % 6;
        const int a = q < 3 ? q : (q == 3 ? 0 : (q == 4 ? 0 : 1));
        const int b = q < 3 ? q : (q == 3 ? 1 : 2);
        double acc = 0.0;
        for (int m = 0; m < N; ++m)
            acc = fma(A[m * N + t], bf3_hess(s, D, m, x + t * 3, R[(t * N + m) * 4], a, b), acc);
        T[t * 6 + q] = acc;
    }
    __syncthreads();
    auto Tab = [&](int t, int a, int b) {
        if (a > b) {
            const int c = a;
            a = b;
            b = c;
        }
        const int q = a == b ? a : (a == 0 ? (b == 1 ? 3 : 4) : 5);
        return T[t * 6 + q];
    };
    // Every particle k's derivatives, one warp per particle (k = warp, warp +
    // NT/32, ...): no block barrier inside.  Each warp's Jacobian columns and
    // their F·∂²x rows (12N) live in R's area, free once G and T are formed,
    // or from J on when R is smaller than 48N (N < 12: the host sizes the
    // area for it).
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* Jw = (N >= 12 ? R : J) + warp * 12 * N;   // [β][t·3 + a] (9N), then F·∂²x [β][t] (3N)
    double* FSw = Jw + 9 * N;
    for (int k = warp; k < np; k += NT / 32) {
        bool hit = k >= D.first && k < D.last;
        for (int c = 0; c < D.nch && !hit; ++c) hit = in_sources(D.ch[c], k);
        if (!hit) continue;
        const double* rk = v.pos + k * 3;
        const int tk = (k >= D.first && k < D.last) ? k - D.first : -1;
        // k's own row: Σ_j B(r_kj) and Σ_j F_k·S(r_kj) over the sources, over the warp
        double own[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (tk >= 0) {
            const double* Fk = F + tk * 3;
            for (int j = lane; j < np; j += 32) {
                if (j == k) continue;
                for (int c = 0; c < D.nch; ++c) {
                    if (!in_sources(D.ch[c], j)) continue;
                    double unused[3] = {0, 0, 0}, B[9], S[9];
                    if (!bf3_pair(s, D.ch[c], rk, v.pos + j * 3, 1.0, unused, B, S)) continue;
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            own[b * 3 + a] += B[a * 3 + b];
                            own[9 + b] += Fk[a] * S[a * 3 + b];
                        }
                }
            }
#pragma unroll
            for (int q = 0; q < 12; ++q) own[q] = warp_sum(own[q]);
        }
        // Jacobian columns Jw[β][t·3 + a] = ∂x_t^a/∂r_k^β and F_t·∂²x_t/∂(r_k^β)², lane = row
        // (N <= 32); nz: row t's column is nonzero (k's own row, or t within a
        // backflow cutoff of k)
        bool nz = false;
        for (int t = lane; t < N; t += 32) {
            double vj[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, fs[3] = {0, 0, 0};
            const double* Ft = F + t * 3;
            nz = t == tk;
            if (t == tk) {
#pragma unroll
                for (int q = 0; q < 9; ++q) vj[q] = own[q] + (q % 4 == 0 ? 1.0 : 0.0);   // [β·3 + a]
                fs[0] = own[9];
                fs[1] = own[10];
                fs[2] = own[11];
            } else {
                const int P = D.first + t;
                for (int c = 0; c < D.nch; ++c) {
                    if (!in_sources(D.ch[c], k)) continue;
                    double unused[3] = {0, 0, 0}, B[9], S[9];
                    if (!bf3_pair(s, D.ch[c], v.pos + P * 3, rk, 1.0, unused, B, S)) continue;
                    nz = true;
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            vj[b * 3 + a] -= B[a * 3 + b];
                            fs[b] += Ft[a] * S[a * 3 + b];
                        }
                }
            }
#pragma unroll
            for (int b = 0; b < 3; ++b) {
#pragma unroll
                for (int a = 0; a < 3; ++a) Jw[b * 3 * N + t * 3 + a] = vj[b * 3 + a];
                FSw[b * N + t] = fs[b];
            }
        }
        __syncwarp();
        // ∂_k ln|D|^β = Σ_t F_t·J_β;  ∂²: Σ F·∂²x + Σ_t J T J - Σ_{j,r} U_jr U_rj, U = Σ_a G^a J^a
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int e = lane; e < 3 * N; e += 32) {
            const int b = e / N, t = e % N;
            const double* vt = Jw + b * 3 * N + t * 3;
            double gg = 0.0, tt = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                gg += F[t * 3 + a] * vt[a];
#pragma unroll
                for (int c = 0; c < 3; ++c) tt += vt[a] * vt[c] * Tab(t, a, c);
            }
            acc[b] += gg;
            acc[3 + b] += tt + FSw[b * N + t];
        }
        // U_jr vanishes with row r's column and U_rj with row j's: the pairs of
        // nonzero rows only, srow on lane i the i-th of them
        const unsigned smask = __ballot_sync(0xffffffffu, nz);
        const int ns = __popc(smask), n2 = ns * ns;
        const unsigned spos = __fns(smask, 0, lane + 1);
        const int srow = spos < 32u ? static_cast<int>(spos) : 0;
        for (int base = 0; base < 3 * n2; base += 32) {   // every lane takes part in the shuffles
            const int e = base + lane;
            const bool on = e < 3 * n2;
            const int ee = on ? e : 0;
            const int b = ee / n2, jr = ee % n2;
            const int j = __shfl_sync(0xffffffffu, srow, jr / ns);
            const int r = __shfl_sync(0xffffffffu, srow, jr % ns);
            if (on) {
                const double* vb = Jw + b * 3 * N;
                double u1 = 0.0, u2 = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    u1 += vb[r * 3 + a] * G[a * N * N + j * N + r];
                    u2 += vb[j * 3 + a] * G[a * N * N + r * N + j];
                }
                acc[3 + b] -= u1 * u2;
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[q] = warp_sum(acc[q]);
        if (lane == 0)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                v.sg[k * 3 + b] += acc[b];
                v.sl[k * 3 + b] += acc[3 + b];
            }
        __syncwarp();
    }
    __syncthreads();
}

// ───────────────────────── local energy ─────────────────────────────────

template <int NT>
__device__ double local_energy3(const DevSys& s, const V3& v) {
    const int np = s.np;
    double acc[1] = {0.0};
    for (int t = threadIdx.x; t < np * 3; t += NT) {
        const double g = v.sg[t] + v.jg[t], l = v.sl[t] + v.jl[t];
        acc[0] += -0.5 * s.inv_mass[t] * (l + g * g);
    }
    const int npair = np * (np - 1) / 2;
    if (s.ewald) {
        for (int q = threadIdx.x; q < npair; q += NT) {
            int i = 0, rem = q;
            while (rem >= np - 1 - i) {
                rem -= np - 1 - i;
                ++i;
            }
            const int j = i + 1 + rem;
            const double coeff = s.charge[i] * s.charge[j];
            if (coeff == 0.0) continue;
            double del[3];
            const double r = dist3(s, v.pos + i * 3, v.pos + j * 3, del);
            if (r < s.e_rcut) acc[0] += coeff * (s.e_inv_eps / r - spline1(s.esp, r));
        }
        for (int k = threadIdx.x; k < s.enk; k += NT) {
            const double kx = s.ek3[k * 3], ky = s.ek3[k * 3 + 1], kz = s.ek3[k * 3 + 2];
            double rr = 0.0, ri = 0.0;
            for (int i = 0; i < np; ++i) {
                const double q = s.charge[i];
                if (q == 0.0) continue;
                double sn, c;
                sincos(fma(kz, v.pos[i * 3 + 2], fma(ky, v.pos[i * 3 + 1], kx * v.pos[i * 3])), &sn, &c);
                rr = fma(q, c, rr);
                ri = fma(q, sn, ri);
            }
            acc[0] += s.ew[k] * (rr * rr + ri * ri);
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
            acc[0] += s.coul_coef[c] / dist3(s, v.pos + i * 3, v.pos + j * 3, del);
        }
    }
    block_sum<NT>(acc, v.red);
    return acc[0] + (s.ewald ? s.e_const : 0.0);
}

// Every particle's derivatives (determinants anew when `invert`, else from
// the committed inverses), ln ψ and E_L into the staged record.
template <int NT>
__device__ void refresh_walker3(const DevSys& s, const V3& v, double* sm, bool invert) {
    const int n3 = s.np * 3;
    for (int i = threadIdx.x; i < n3; i += NT) v.sg[i] = v.sl[i] = v.kg[i] = v.kl[i] = 0.0;
    __syncthreads();
    for (int d = 0; d < s.nbf; ++d) bf3_refresh<NT>(s, v, sm, d, invert);
    __syncthreads();
    const double lj = jastrow_all<NT>(s, v);
    const double el = local_energy3<NT>(s, v);
    if (threadIdx.x == 0) {
        double lp = lj;
        for (int d = 0; d < s.nbf; ++d) lp += sm[s.bf[d].oLS];
        v.scal[S_LOGPSI] = lp;
        v.scal[S_EL] = el;
    }
    __syncthreads();
}

// ───────────────────────── one move ─────────────────────────────────────

__device__ __forceinline__ bool bf_touches(const DevBF& D, int k) {
    if (k >= D.first && k < D.last) return true;
    for (int c = 0; c < D.nch; ++c)
        if (in_sources(D.ch[c], k)) return true;
    return false;
}

// The pair terms' change of ln J when p moves to v.newpos, for the partner
// j, and the partner's share of p's new Jastrow gradient and per-dimension
// Laplacian: acc[0] += Δu, acc[1..3] += u'(r') r̂', acc[4..6] += u'' r̂_d² +
// u'/r (1 - r̂_d²).
__device__ __forceinline__ void jastrow_pair_change(const DevSys& s, const V3& v, int p, int j, double* acc) {
    for (int t = 0; t < s.nterms; ++t) {
        const DevTerm& T = s.terms[t];
        if (!any_term_couples(T, p, j)) continue;
        double del[3], u, du, d2u;
        const double ro = dist3(s, v.pos + p * 3, v.pos + j * 3, del);
        radial(T, ro, u, du, d2u);
        acc[0] -= u;
        const double rn = dist3(s, v.newpos, v.pos + j * 3, del);
        radial(T, rn, u, du, d2u);
        acc[0] += u;
        const double ir = 1.0 / rn;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double dor = del[d] * ir;
            acc[1 + d] += du * dor;
            acc[4 + d] += d2u * dor * dor + du * ir * (1.0 - dor * dor);
        }
    }
}

// The proposal of p for every determinant it touches: pending x', A', F',
// (log|det|', sign', regular) in each one's pending area; with `grad`, the
// determinants' part of p's new gradient is added to misc[T_GN..].  The
// phases run over the CTA for all touched determinants together, the
// inversions on one warp per determinant (warp d inverts determinant d).
// Move work area per determinant: ∇φ rows [(t·N + m)·3 + a] (3N²), the
// Gauss-Jordan multipliers (N) and row exchanges (N ints).  While warps 0
// and 1 invert, warps 2 and 3 form the Jastrow ratio and p's new Jastrow
// gradient into misc (with fewer warps ratio3 forms them first).  The ∇φ
// rows are not kept (the moves' layout fits four walkers per SM): F'
// evaluates them again, two lanes per row.  Move work area per determinant:
// the Gauss-Jordan multipliers (N) and row exchanges (N ints).  (Keeping the
// new orbital values for F', a plane wave's gradient being its partner's
// value times ±k, ran no faster in 12 KB more per walker.)
template <int NT>
__device__ void propose3(const DevSys& s, const V3& v, double* sm, const unsigned char (*units)[33], int p,
                         bool grad) {
    const int np = s.np, nb = s.nbf, W = s.maxN;
    const long mstride = (2L * W + 3) & ~3L;
    bool touched[2] = {false, false};
    int dp = -1;
    for (int d = 0; d < nb; ++d) {
        touched[d] = bf_touches(s.bf[d], p);
        if (p >= s.bf[d].first && p < s.bf[d].last) dp = d;
    }
    // p's own row, r_p' + Σ_c Σ_j η(r_pj') r_pj' over the sources, on the last
    // warp, while the others shift the rows that p displaces (the committed x
    // moved by p's old and new pair terms)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int NW = NT / 32;
    const bool own_warp = NW > 1 && dp >= 0 && warp == NW - 1;
    if (own_warp) {
        const DevBF& D = s.bf[dp];
        double acc[3] = {0.0, 0.0, 0.0};
        for (int j = lane; j < np; j += 32) {
            if (j == p) continue;
            for (int c = 0; c < D.nch; ++c)
                if (in_sources(D.ch[c], j)) bf3_pair(s, D.ch[c], v.newpos, v.pos + j * 3, 1.0, acc, nullptr, nullptr);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] = warp_sum(acc[a]);
        if (lane == 0) {
            double* px = sm + D.pX + (p - D.first) * 3;
            px[0] = v.newpos[0] + acc[0];
            px[1] = v.newpos[1] + acc[1];
            px[2] = v.newpos[2] + acc[2];
        }
    } else if (NW == 1 && dp >= 0 && threadIdx.x == 0) {   // a one-warp CTA: serially
        const DevBF& D = s.bf[dp];
        double xt[3] = {v.newpos[0], v.newpos[1], v.newpos[2]};
        for (int j = 0; j < np; ++j) {
            if (j == p) continue;
            for (int c = 0; c < D.nch; ++c)
                if (in_sources(D.ch[c], j)) bf3_pair(s, D.ch[c], v.newpos, v.pos + j * 3, 1.0, xt, nullptr, nullptr);
        }
        double* px = sm + D.pX + (p - D.first) * 3;
        px[0] = xt[0];
        px[1] = xt[1];
        px[2] = xt[2];
    }
    const int shifters = (NW > 1 && dp >= 0) ? NT - 32 : NT;
    if (!own_warp)
        for (int e = threadIdx.x; e < nb * W; e += shifters) {
            const int d = e / W, t = e % W;
            const DevBF& D = s.bf[d];
            const int P = D.first + t;
            if (!touched[d] || t >= D.n || P == p) continue;
            const double* x = sm + D.oX;
            double xt[3] = {x[t * 3], x[t * 3 + 1], x[t * 3 + 2]};
            for (int c = 0; c < D.nch; ++c) {
                if (!in_sources(D.ch[c], p)) continue;
                bf3_pair(s, D.ch[c], v.pos + P * 3, v.newpos, 1.0, xt, nullptr, nullptr);
                bf3_pair(s, D.ch[c], v.pos + P * 3, v.pos + p * 3, -1.0, xt, nullptr, nullptr);
            }
            double* px = sm + D.pX + t * 3;
            px[0] = xt[0];
            px[1] = xt[1];
            px[2] = xt[2];
        }
    __syncthreads();
    // the new matrices (values into A's pending storage, inverted there), one
    // work item per orbital unit of a row (units: a plane wave's cosine and
    // sine of one k take one sincos)
    const int U = max(static_cast<int>(units[0][32]), nb > 1 ? static_cast<int>(units[1][32]) : 0);
    for (int e = threadIdx.x; e < nb * W * U; e += NT) {
        const int d = e / (W * U), tu = e % (W * U), t = tu / U, u = tu % U;
        const DevBF& D = s.bf[d];
        if (!touched[d] || t >= D.n || u >= units[d][32]) continue;
        const int N = D.n, mu = units[d][u], m = mu & 31;
        const double* xt = sm + D.pX + t * 3;
        double* row = sm + D.pA + t * N;
        if (D.type == 0) {
            const double* k = D.k + m * 3;
            double sn, c;
            sincos(fma(k[2], xt[2], fma(k[1], xt[1], k[0] * xt[0])), &sn, &c);
            row[m] = D.is_sin[m] != 0.0 ? sn : c;
            if (mu & kUnitPair) row[m + 1] = sn;
        } else {
            double val, g[3];
            bf3_orbital(s, D, m, xt, val, g);
            row[m] = val;
        }
    }
    __syncthreads();
    if (warp < nb && touched[warp]) {
        const DevBF& D = s.bf[warp];
        double* mult = v.mwork + warp * mstride;
        gj_warp_signed(sm + D.pA, D.n, mult, reinterpret_cast<int*>(mult + D.n), sm + D.pM);
    } else if (NT >= 128 && warp >= 2) {
        // meanwhile warps 2 and 3: the Jastrow ratio and p's new Jastrow
        // gradient and Laplacian, each warp's partial sums to v.red[64 + 8·(warp - 2)..]
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int j = threadIdx.x - 64; j < np; j += 64) {
            if (j == p) continue;
            jastrow_pair_change(s, v, p, j, acc);
        }
#pragma unroll
        for (int q = 0; q < 7; ++q) acc[q] = warp_sum(acc[q]);
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int q = 0; q < 7; ++q) v.red[64 + 8 * (warp - 2) + q] = acc[q];
    }
    __syncthreads();
    if (NT >= 128 && threadIdx.x == 0) {
        v.misc[T_LOGR] = v.red[64] + v.red[72];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v.misc[T_JG + d] = v.misc[T_GN + d] = v.red[65 + d] + v.red[73 + d];
            v.misc[T_JL + d] = v.red[68 + d] + v.red[76 + d];
        }
    }
    // F'_t = Σ_m A'[m][t] ∇φ_m(x'_t)
    // lanes 2i and 2i + 1 take the even and odd orbital units (plane waves) or
    // orbitals of one row; every lane of the warp takes part in the pair's
    // shuffle
    for (int base = 0; base < nb * W * 2; base += NT) {
        const int e = base + threadIdx.x, h = e & 1, dt = e >> 1, d = dt / W, t = dt % W;
        const DevBF* Dp = d < nb ? &s.bf[d] : nullptr;
        const bool on = e < nb * W * 2 && touched[d] && t < Dp->n && sm[Dp->pM + 2] != 0.0;
        double acc[3] = {0.0, 0.0, 0.0};
        if (on) {
            const DevBF& D = *Dp;
            const int N = D.n;
            const double* pa = sm + D.pA;
            const double* xt = sm + D.pX + t * 3;
            if (D.type == 0) {   // by orbital units: one sincos per cosine-sine pair
                for (int u = h; u < units[d][32]; u += 2) {
                    const int mu = units[d][u], m = mu & 31;
                    const double* k = D.k + m * 3;
                    double sn, c;
                    sincos(fma(k[2], xt[2], fma(k[1], xt[1], k[0] * xt[0])), &sn, &c);
                    const double dv = D.is_sin[m] != 0.0 ? c : -sn;
                    const double am = pa[m * N + t];
#pragma unroll
                    for (int a = 0; a < 3; ++a) acc[a] = fma(am, k[a] * dv, acc[a]);
                    if (mu & kUnitPair) {
                        const double an = pa[(m + 1) * N + t];
#pragma unroll
                        for (int a = 0; a < 3; ++a) acc[a] = fma(an, k[a] * c, acc[a]);
                    }
                }
            } else {
                for (int m = h; m < N; m += 2) {
                    double val, g[3];
                    bf3_orbital(s, D, m, xt, val, g);
                    const double am = pa[m * N + t];
                    acc[0] = fma(am, g[0], acc[0]);
                    acc[1] = fma(am, g[1], acc[1]);
                    acc[2] = fma(am, g[2], acc[2]);
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], 1);
        if (on && h == 0) {
            double* pf = sm + Dp->pF + t * 3;
            pf[0] = acc[0];
            pf[1] = acc[1];
            pf[2] = acc[2];
        }
    }
    __syncthreads();
    if (grad)
        for (int d = 0; d < nb; ++d) {
            const DevBF& D = s.bf[d];
            if (!touched[d] || sm[D.pM + 2] == 0.0) continue;
            double g[3];
            bf3_grad<NT>(s, D, sm + D.pF, v.pos, p, p, v.newpos, v.red, g);
            if (threadIdx.x == 0) {
                v.misc[T_GN] += g[0];
                v.misc[T_GN + 1] += g[1];
                v.misc[T_GN + 2] += g[2];
            }
            __syncthreads();
        }
}

// log ψ(R')/ψ(R), its sign and (with grad) p's new gradient, for the
// proposal in v.newpos, in thread 0's misc slots: the caller's next barrier
// publishes them.  Called after a barrier.
template <int NT>
__device__ void ratio3(const DevSys& s, const V3& v, double* sm, const unsigned char (*units)[33], int p,
                       bool grad) {
    if (threadIdx.x == 0) {
        v.misc[T_SIGN] = 1.0;
        v.misc[T_BAD] = 0.0;
    }
    if constexpr (NT < 128) {   // no spare warps during the inversions: the Jastrow first
        double acc[7] = {0, 0, 0, 0, 0, 0, 0};
        for (int j = threadIdx.x; j < s.np; j += NT)
            if (j != p) jastrow_pair_change(s, v, p, j, acc);
        block_sum<NT>(acc, v.red);
        if (threadIdx.x == 0) {
            v.misc[T_LOGR] = acc[0];
            for (int d = 0; d < 3; ++d) {
                v.misc[T_JG + d] = v.misc[T_GN + d] = acc[1 + d];
                v.misc[T_JL + d] = acc[4 + d];
            }
        }
        __syncthreads();
    }
    // (T_SIGN and T_BAD are thread 0's alone until the caller's next barrier)
    propose3<NT>(s, v, sm, units, p, grad);
    if (threadIdx.x == 0)
        for (int d = 0; d < s.nbf; ++d) {
            const DevBF& D = s.bf[d];
            if (!bf_touches(D, p)) continue;
            const double* pm = sm + D.pM;
            const double* ls = sm + D.oLS;
            if (pm[2] == 0.0) {
                v.misc[T_BAD] = 1.0;
            } else {
                v.misc[T_LOGR] += pm[0] - ls[0];
                v.misc[T_SIGN] *= pm[1] * ls[1];
            }
        }
}

// Accepted move of p: position (wrapped), pending determinants, the Jastrow
// planes of p and its partners.  p's new position is thread 0's store after
// the last barrier; with sync_pos a barrier publishes it (the drift moves'
// refresh of the next particle reads every position), else the caller's
// next barrier does.
template <int NT>
__device__ void commit3(const DevSys& s, const V3& v, double* sm, int p, bool sync_pos) {
    const int np = s.np;
    for (int j = threadIdx.x; j < np; j += NT) {
        if (j == p) continue;
        double dg[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
        bool any = false;
        for (int t = 0; t < s.nterms; ++t) {
            const DevTerm& T = s.terms[t];
            if (!any_term_couples(T, p, j)) continue;
            any = true;
            for (int side = 0; side < 2; ++side) {
                double del[3], u, du, d2u;
                const double r = dist3(s, v.pos + j * 3, side ? v.newpos : v.pos + p * 3, del);
                radial(T, r, u, du, d2u);
                const double sg = side ? 1.0 : -1.0, ir = 1.0 / r;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double dor = del[d] * ir;
                    dg[d] += sg * du * dor;
                    dl[d] += sg * (d2u * dor * dor + du * ir * (1.0 - dor * dor));
                }
            }
        }
        if (any)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v.jg[j * 3 + d] += dg[d];
                v.jl[j * 3 + d] += dl[d];
            }
    }
    // p's own planes: the proposal's sums over its new partners
    if (threadIdx.x == 0)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v.jg[p * 3 + d] = v.misc[T_JG + d];
            v.jl[p * 3 + d] = v.misc[T_JL + d];
        }
    for (int d = 0; d < s.nbf; ++d) {
        const DevBF& D = s.bf[d];
        if (!bf_touches(D, p)) continue;
        const int N = D.n;
        for (int e = threadIdx.x; e < 3 * N; e += NT) {
            sm[D.oX + e] = sm[D.pX + e];
            sm[D.oF + e] = sm[D.pF + e];
        }
        for (int e = threadIdx.x; e < N * N; e += NT) sm[D.oA + e] = sm[D.pA + e];
        if (threadIdx.x == 0) {
            sm[D.oLS] = sm[D.pM];
            sm[D.oLS + 1] = sm[D.pM + 1];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r[3] = {v.newpos[0], v.newpos[1], v.newpos[2]};
        wrap_pos(s, r);
        v.pos[p * 3] = r[0];
        v.pos[p * 3 + 1] = r[1];
        v.pos[p * 3 + 2] = r[2];
    }
    if (sync_pos) __syncthreads();
}

// The determinant part of p's gradient at the committed state into sg
// (refresh_particle_derivatives).
template <int NT>
__device__ void refresh_particle3(const DevSys& s, const V3& v, double* sm, int p) {
    double tot[3] = {0, 0, 0};
    for (int d = 0; d < s.nbf; ++d) {
        const DevBF& D = s.bf[d];
        if (!bf_touches(D, p)) continue;
        double g[3];
        bf3_grad<NT>(s, D, sm + D.oF, v.pos, p, -1, nullptr, v.red, g);
        tot[0] += g[0];
        tot[1] += g[1];
        tot[2] += g[2];
    }
    if (threadIdx.x == 0) {
        v.sg[p * 3] = tot[0];
        v.sg[p * 3 + 1] = tot[1];
        v.sg[p * 3 + 2] = tot[2];
    }
    __syncthreads();
}

// ───────────────────────── record staging ───────────────────────────────
//
// A walker's record is contiguous and all of it is hot, so it moves between
// HBM and shared memory as one bulk copy of the tensor-memory-access engine
// (cp.async.bulk, no tensor map): thread 0 arms an mbarrier with the byte
// count and issues the load; every thread waits on the barrier's phase, the
// wait bounded (about a second) so that a copy that never lands sets the
// walker's error flag instead of hanging the kernel.  The store back is a
// bulk copy of the staged record after the generic-proxy writes are fenced
// for the async proxy.  Record strides and the hot size are multiples of 32
// bytes, the shared base of 16: the alignment both copies need.

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// true when the record landed; false after the bounded wait ran out
__device__ bool stage_in(const double* rec, double* sm, unsigned bytes, unsigned long long* bar) {
    const unsigned b = smem_addr(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_addr(sm)), "l"(rec), "r"(bytes), "r"(b)
                     : "memory");
    }
    auto wait = [b](long limit) {
        unsigned done = 0;
        for (long it = 0; it < limit && !done; ++it)
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"(done)
                : "r"(b)
                : "memory");
        return done != 0;
    };
    if (__syncthreads_and(wait(1L << 24))) return true;
    wait(1L << 24);   // the copy still in flight: a second bounded wait before the CTA leaves
    __syncthreads();
    return false;
}

__device__ void stage_out(double* rec, const double* sm, unsigned bytes) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(rec), "r"(smem_addr(sm)),
                     "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    __syncthreads();
}

// ───────────────────────── kernels ──────────────────────────────────────

template <int NT>
__global__ void __launch_bounds__(NT) evaluate3_kernel(DevSys s, double* records, int nw) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    __shared__ unsigned long long bar;
    if (!stage_in(rec, sm, static_cast<unsigned>(s.hot) * 8u, &bar)) {
        if (threadIdx.x == 0) rec[s.o_scal + S_ERR] = 2.0;   // the record never landed
        return;
    }
    const V3 v = view3(s, sm);
    if (threadIdx.x == 0) v.misc[T_ERR] = 0.0;
    for (int i = threadIdx.x; i < s.np; i += NT) wrap_pos(s, v.pos + i * 3);
    __syncthreads();
    refresh_walker3<NT>(s, v, sm, true);
    if (threadIdx.x == 0) v.scal[S_ERR] = v.misc[T_ERR];
    stage_out(rec, sm, static_cast<unsigned>(s.hot) * 8u);
}

// The moves of prm.n_sub sweeps, in the moves' shared-memory layout (four
// walkers per SM); the host follows each DMC sweep, or a VMC step's sweeps,
// with refresh3_kernel (derivatives, E_L, branch factor).  `first` marks a
// step's first launch: its scalars start there.
template <int NT>
__global__ void __launch_bounds__(NT, 4) sweep3_kernel(DevSys s, double* records, int nw, const double* randoms,
                                                       long stride, SweepParams prm, int first) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    __shared__ unsigned long long bar;
    if (!stage_in(rec, sm, static_cast<unsigned>(s.hot) * 8u, &bar)) {
        if (threadIdx.x == 0) rec[s.o_scal + S_ERR] = 2.0;   // the record never landed
        return;
    }
    const V3 v = view3(s, sm);
    const int np = s.np;
    const bool dmc = prm.mode == 1;
    const bool drift = dmc || prm.drift != 0;
    if (threadIdx.x == 0 && first) {
        v.scal[S_NACC] = 0.0;
        v.scal[S_NCUT] = 0.0;
        if (dmc) {
            v.scal[S_RRP] = 0.0;
            v.scal[S_RRA] = 0.0;
            v.scal[S_WEIGHT] = 1.0;
            v.scal[S_EPREV] = v.scal[S_EL];
        }
    }
    if (threadIdx.x == 0) v.misc[T_ERR] = 0.0;
    __shared__ unsigned char units[2][33];
    build_units(s, units);
    __syncthreads();
    for (int sub = 0; sub < prm.n_sub; ++sub) {
        const double* rnd = randoms + static_cast<long>(sub) * np * 4 * stride;
        for (int p = 0; p < np; ++p) {
            if (drift) refresh_particle3<NT>(s, v, sm, p);
            if (threadIdx.x == 0) {
                const double* g = rnd + static_cast<long>(p) * 4 * stride;
                double go[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) go[d] = v.sg[p * 3 + d] + v.jg[p * 3 + d];
                const double tm = prm.tau * s.inv_mass[p * 3];
                double sc = tm;
                if (dmc) {
                    const double vsq = go[0] * go[0] + go[1] * go[1] + go[2] * go[2];
                    sc = vsq < 1e-10 ? tm : (-1.0 + sqrt(1.0 + 2.0 * tm * vsq)) / vsq;
                }
                v.misc[T_SCF] = sc;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double sig = prm.sigma[p * 3 + d];
                    const double td = dmc ? sc : prm.tau * s.inv_mass[p * 3 + d];
                    v.newpos[d] = drift ? fma(sig, g[d * stride + w], fma(td, go[d], v.pos[p * 3 + d]))
                                        : fma(sig, g[d * stride + w], v.pos[p * 3 + d]);
                    v.misc[T_GO + d] = go[d];
                }
                v.misc[T_U] = g[3 * stride + w];
            }
            __syncthreads();
            ratio3<NT>(s, v, sm, units, p, drift);
            if (threadIdx.x == 0) {
                const double logr = v.misc[T_LOGR];
                const double u = v.misc[T_U];
                const bool bad = v.misc[T_BAD] != 0.0;
                double dx[3], tmd[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    dx[d] = v.newpos[d] - v.pos[p * 3 + d];
                    tmd[d] = prm.tau * s.inv_mass[p * 3 + d];
                }
                const double* go = v.misc + T_GO;
                const double* gn = v.misc + T_GN;
                bool acc = false;
                if (dmc) {
                    if (!bad && v.misc[T_SIGN] > 0.0) {
                        const double vsq = gn[0] * gn[0] + gn[1] * gn[1] + gn[2] * gn[2];
                        const double sb = vsq < 1e-10 ? tmd[0] : (-1.0 + sqrt(1.0 + 2.0 * tmd[0] * vsq)) / vsq;
                        const double sf = v.misc[T_SCF];
                        double lc = 0.0;
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            if (tmd[d] > 0.0) {
                                const double df = sf * go[d], db = sb * gn[d];
                                lc += (-dx[d] * (df + db) + 0.5 * (df * df - db * db)) / tmd[d];
                            }
                        const double la = 2.0 * logr + lc;
                        acc = la >= 0.0 || u < exp(la);
                    }
                    double rr = 0.0;
#pragma unroll
                    for (int d = 0; d < 3; ++d) rr += tmd[d] * dx[d] * dx[d];
                    v.scal[S_RRP] += rr;
                    if (acc) v.scal[S_RRA] += rr;
                } else if (bad) {
                    acc = false;
                } else if (prm.drift) {
                    double lc = 0.0;
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        lc += -dx[d] * (go[d] + gn[d]) + 0.5 * tmd[d] * (go[d] * go[d] - gn[d] * gn[d]);
                    const double la = 2.0 * logr + lc;
                    acc = la >= 0.0 || u < exp(la);
                } else {
                    acc = u < exp(2.0 * logr);
                }
                v.misc[T_ACC] = acc ? 1.0 : 0.0;
                if (acc) v.scal[S_NACC] += 1.0;
            }
            __syncthreads();
            if (v.misc[T_ACC] != 0.0) commit3<NT>(s, v, sm, p, drift);
        }
    }
    if (threadIdx.x == 0 && v.misc[T_ERR] != 0.0) v.scal[S_ERR] = 1.0;
    stage_out(rec, sm, static_cast<unsigned>(s.hot) * 8u);
}

// After a moves-only launch: every particle's derivatives from the committed
// state, ln ψ and E_L; in DMC the branch factor of the sweep, and after the
// step's last sweep the age (the fused kernel's end of a sweep).
template <int NT>
__global__ void __launch_bounds__(NT, 3) refresh3_kernel(DevSys s, double* records, int nw, SweepParams prm,
                                                        int last) {
    extern __shared__ __align__(16) double sm[];
    const int w = blockIdx.x;
    if (w >= nw) return;
    double* rec = records + static_cast<long>(w) * s.rec;
    __shared__ unsigned long long bar;
    if (!stage_in(rec, sm, static_cast<unsigned>(s.hot) * 8u, &bar)) {
        if (threadIdx.x == 0) rec[s.o_scal + S_ERR] = 2.0;   // the record never landed
        return;
    }
    const V3 v = view3(s, sm);
    const bool dmc = prm.mode == 1;
    if (threadIdx.x == 0) v.misc[T_ERR] = 0.0;
    __syncthreads();
    refresh_walker3<NT>(s, v, sm, false);
    if (threadIdx.x == 0) {
        if (dmc) {
            const double enew = v.scal[S_EL], eold = v.scal[S_EPREV];
            double half_tau = 0.5 * prm.tau;
            const double x = fmax(prm.eref - enew, prm.eref - eold);
            if (x > prm.e_max)
                half_tau = 0.0;
            else if (x > prm.e_cut)
                half_tau *= 1.0 - (x - prm.e_cut) / (prm.e_max - prm.e_cut);
            v.scal[S_WEIGHT] *= exp(half_tau * (2.0 * prm.etrial - enew - eold));
            if (x > prm.e_cut) v.scal[S_NCUT] += 1.0;
            v.scal[S_EPREV] = enew;
            if (last && prm.tau > 0.0) v.scal[S_AGE] = v.scal[S_RRP] > 0.0 ? 0.0 : v.scal[S_AGE] + 1.0;
        }
        if (v.misc[T_ERR] != 0.0) v.scal[S_ERR] = 1.0;
    }
    stage_out(rec, sm, static_cast<unsigned>(s.hot) * 8u);
}

}  // namespace

cudaError_t launch_evaluate3(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records) {
    const cudaError_t e = cudaFuncSetAttribute(evaluate3_kernel<kNT3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    evaluate3_kernel<kNT3><<<nw, kNT3, smem, st>>>(s, records, nw);
    return cudaGetLastError();
}

// The moves run as their own launches (four walkers per SM in the moves'
// layout, s.t_mtotal doubles) followed by refresh3_kernel (the full layout):
// one moves launch for a VMC step's sweeps, one pair per DMC sweep.
cudaError_t launch_sweep3(int nw, size_t smem, cudaStream_t st, const DevSys& s, double* records,
                          const double* randoms, long stride, const SweepParams& prm) {
    const size_t msmem = static_cast<size_t>(s.t_mtotal) * 8;
    cudaError_t e = cudaFuncSetAttribute(sweep3_kernel<kNT3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(msmem));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(refresh3_kernel<kNT3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const bool dmc = prm.mode == 1;
    const int launches = dmc ? prm.n_sub : 1;
    for (int l = 0; l < launches; ++l) {
        SweepParams mp = prm;
        mp.n_sub = dmc ? 1 : prm.n_sub;
        const double* rnd = randoms + static_cast<long>(dmc ? l : 0) * s.np * 4 * stride;
        sweep3_kernel<kNT3><<<nw, kNT3, msmem, st>>>(s, records, nw, rnd, stride, mp, l == 0 ? 1 : 0);
        refresh3_kernel<kNT3><<<nw, kNT3, smem, st>>>(s, records, nw, prm, l == launches - 1 ? 1 : 0);
    }
    return cudaGetLastError();
}

}  // namespace alea_gpu
