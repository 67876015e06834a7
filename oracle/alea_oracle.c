/*
 * Oracle: a plain-C restatement of the reference's VMC/DMC walker hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker;
 * the product never links or calls it.
 *
 * It restates, walker by walker and in the reference's order of operations,
 * the algorithms of ItaloAlb/alea (paths relative to the reference tree):
 *   RNG              src/numerics/xoshiro_random.h:23-49, :90-108, :183-189;
 *                    src/numerics/random.h:39-56
 *   sweep randoms    src/qmc/sweep_blocking.h:39-48
 *   cell             src/population/simulation_cell.h:109-189, :224-261
 *   distances        src/population/batched_distance_table.cpp:20-101
 *   orbitals         src/wavefunction/orbital_set.h:185-224 (Gaussian),
 *                    :436-474 (plane waves)
 *   Slater           src/wavefunction/slater_determinant.cpp:305-437 (evaluate,
 *                    ratio), :515-726 (Sherman-Morrison commit, walker-tile
 *                    path), :862-903 (refresh), :905-993 (Gauss-Jordan)
 *   pair Jastrows    src/wavefunction/pade_jastrow.cpp:24-60, :250-634;
 *                    src/wavefunction/radial_pair_jastrow_impl.h;
 *                    src/wavefunction/drummond_jastrow.cpp (DTN u(r))
 *   image sum        src/wavefunction/periodic_pair_sum.cpp:62-80 (short range),
 *                    src/wavefunction/kspace_pair_sum.cpp (rho(k), ratio, accept),
 *                    src/numerics/reciprocal_phases.h (ladders),
 *                    src/numerics/long_range_spline.h:41-135
 *   Hamiltonian      src/hamiltonian/kinetic.cpp:45-72,
 *                    src/hamiltonian/ewald_term.cpp:368-612,
 *                    src/hamiltonian/coulomb.cpp:31-61
 *   drivers          src/qmc/vmc.cpp:23-431, src/qmc/dmc.cpp:203-884,
 *                    src/qmc/population_control.cpp:37-103,
 *                    src/population/walker_set.cpp:187-239 (branch),
 *                    src/numerics/green_function.h:20-58
 *
 * Every sum over particles, orbitals or k-vectors is sequential.  The
 * reference vectorises some of them with `omp simd reduction` (the k-space
 * sums), so those agree to rounding only; everything else follows its
 * operations one for one.
 *
 * The system (cell, groups, orbital blocks, pair terms with their breakup
 * tables, Ewald tables) arrives as one flat float64 "blob" whose layout is
 * documented at blob_read().  Parity is pinned against the compiled reference
 * (oracle/_ref) by the tests.
 */
#define _GNU_SOURCE
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXG 8   /* groups */
#define MAXB 4   /* determinant blocks */
#define MAXT 8   /* pair terms (Padé / Drummond) */
#define MAXC 8   /* open Coulomb terms */
#define MAXPAIR 4
#define BF_MAXE (64 * 256)   /* rows x particles of one backflow determinant's pair tables */

/* ───────────────────────── random numbers ───────────────────────────── */

uint64_t o_splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

uint64_t o_stream_seed(uint64_t base, uint64_t stream, uint64_t index) {
    return o_splitmix64(o_splitmix64(o_splitmix64(base) ^ stream) ^ index);
}

typedef struct { uint64_t s[4]; } xo_t;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static void xo_seed(xo_t* r, uint64_t seed) {
    for (uint64_t i = 0; i < 4; ++i) r->s[i] = o_splitmix64(seed + i * 0x9e3779b97f4a7c15ULL);
}

static uint64_t xo_next(xo_t* r) {
    uint64_t* s = r->s;
    const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return result;
}

static double xo_uniform(xo_t* r) {
    return (double)(int64_t)(xo_next(r) >> 11) * 0x1.0p-53;
}

/* Ziggurat tables, built as the reference builds them (bisection for r). */
static struct {
    uint64_t k[256];
    double w[256], f[256], r;
    int ready;
} zig;

static double zf(double x) { return exp(-0.5 * x * x); }
static double zv(double r) {
    return r * zf(r) + sqrt(0.5 * 3.14159265358979323846) * erfc(r / 1.41421356237309504880);
}
static double zig_x[256];
static double zig_mismatch(double r) {
    const double v = zv(r);
    zig_x[255] = r;
    for (int i = 255; i >= 2; --i) {
        const double y = zf(zig_x[i]) + v / zig_x[i];
        if (y >= 1.0) return 1.0;
        zig_x[i - 1] = sqrt(-2.0 * log(y));
    }
    return zf(zig_x[1]) + v / zig_x[1] - 1.0;
}
static void zig_build(void) {
    if (zig.ready) return;
    double lo = 3.0, hi = 4.5;
    for (;;) {
        const double mid = 0.5 * (lo + hi);
        if (mid == lo || mid == hi) break;
        if (zig_mismatch(mid) > 0.0) lo = mid; else hi = mid;
    }
    zig.r = hi;
    (void)zig_mismatch(zig.r);
    const double two52 = 0x1.0p52;
    const double base = zv(zig.r) / zf(zig.r);
    zig.k[0] = (uint64_t)(two52 * (zig.r / base));
    zig.w[0] = base / two52;
    zig.f[0] = 1.0;
    for (int i = 1; i < 256; ++i) {
        zig.k[i] = i == 1 ? 0 : (uint64_t)(two52 * (zig_x[i - 1] / zig_x[i]));
        zig.w[i] = zig_x[i] / two52;
        zig.f[i] = zf(zig_x[i]);
    }
    zig.ready = 1;
}

static double with_sign(double x, uint64_t sign) {
    uint64_t u;
    memcpy(&u, &x, 8);
    u ^= sign;
    memcpy(&x, &u, 8);
    return x;
}

static double xo_gaussian(xo_t* r) {
    for (;;) {
        const uint64_t bits = xo_next(r);
        const unsigned i = (unsigned)(bits & 0xff);
        const uint64_t sign = (bits & 0x100) << 55;
        const uint64_t position = (bits >> 9) & ((1ULL << 52) - 1);
        const double x = (double)(int64_t)position * zig.w[i];
        if (position < zig.k[i]) return with_sign(x, sign);
        if (i == 0) {
            for (;;) {
                const double xi = -log1p(-xo_uniform(r)) / zig.r;
                const double y = -log1p(-xo_uniform(r));
                if (y + y > xi * xi) return with_sign(zig.r + xi, sign);
            }
        }
        if (zig.f[i] + xo_uniform(r) * (zig.f[i - 1] - zig.f[i]) < exp(-0.5 * x * x))
            return with_sign(x, sign);
    }
}

/* Test hooks: raw outputs of a stream from a given state or seed. */
void o_xoshiro_raw(const uint64_t* state, long n, uint64_t* out) {
    xo_t r;
    memcpy(r.s, state, 32);
    for (long i = 0; i < n; ++i) out[i] = xo_next(&r);
}
void o_rng_draws(uint64_t seed, long n, int kind, double* out) {
    zig_build();
    xo_t r;
    xo_seed(&r, seed);
    for (long i = 0; i < n; ++i) out[i] = kind == 0 ? xo_uniform(&r) : xo_gaussian(&r);
}
void o_ziggurat_tables(uint64_t* k, double* w, double* f, double* rr) {
    zig_build();
    memcpy(k, zig.k, sizeof zig.k);
    memcpy(w, zig.w, sizeof zig.w);
    memcpy(f, zig.f, sizeof zig.f);
    *rr = zig.r;
}

/* ───────────────────────── system description ───────────────────────── */

typedef struct { double r_cut, inv_delta; int n_knots; const double* scaled; } spline_t;

typedef struct {
    int kind;                      /* 0 Padé, 1 Drummond */
    int npairs, pairs[MAXPAIR][4]; /* a_first, a_last, b_first, b_last */
    int nnum, nden; double coef[16];
    int image; spline_t sp; double u_inf;
    int nk, m1, m2; const double *n1, *n2, *kx, *ky, *w; double *kx2, *ky2;
    int C; double gamma, L, alpha1; int ncoef; double dc[16];
    int n_cached;                  /* k-space phase-cache rows */
    /* kind 2, zero-energy (zero_energy_jastrow.cpp): s, kappa, R_m, r_c and the
       matching constants; Chebyshev coefficients of sqrt(x) e^x K_{0,1}(x) */
    double ze_s, ze_kappa, ze_rm, ze_rc, ze_c3, ze_logc1, ze_logc2;
    const double* ze_cheb;         /* [2 * 24]: order 0, then order 1 */
} term_t;

/* One backflow channel: sources [sf, sl) displace every row by η(r) r,
 * η = (1 - r/L)^C Σ_k c_k r^k (backflow_function.h; c_1 already derived for
 * a like-spin channel). */
typedef struct { int sf, sl, C; double L; int nc; double c[16]; } bfch_t;

/* A backflow determinant over the rows [first, last) of one group
 * (backflow_slater_determinant.h): one orbital block, its channels, and the
 * walker-record offsets of x (quasi-coordinates), A = M⁻¹, F = A^T ∇φ(x)
 * and (log|det|, sign). */
typedef struct {
    int first, last, type;
    const double *k, *is_sin, *centers, *alphas;
    int nch; bfch_t ch[4];
    long o_x, o_A, o_F, o_ls;
} bfdet_t;

typedef struct {
    int first, last, type;         /* type 0 plane waves, 1 Gaussians, 2 twisted plane waves */
    const double *k, *is_sin, *centers, *alphas;   /* type 2: k holds q = k + θ */
} block_t;

typedef struct {
    int dim, np;
    int periodic, ortho;
    double a[9], ainv[9], recip[9], box[3], inv_box[3], cand[27 * 3];
    int ncand;
    int ngroups, gfirst[MAXG], glast[MAXG];
    double gcharge[MAXG];
    double* inv_mass;              /* [np*dim] */
    double* charge;                /* [np] */
    int nblocks; block_t blocks[MAXB];
    int cplx;                      /* the determinant is complex (twisted plane waves) */
    int nterms; term_t terms[MAXT];
    int ewald; spline_t esp; double e_rcut, e_inv_eps, e_const; int enk, en1max, en2max;
    const double *en1, *en2, *ew;
    int ncoul; int coul[MAXC][4]; double coul_coef[MAXC];
    /* inverse-power pair terms (inverse_power.cpp): pair ranges, C, p, integer p
       (0 when not a small integer), and the sum of their continuum tails */
    int nip; int ip[MAXC][4]; double ip_c[MAXC], ip_p[MAXC]; int ip_pint[MAXC];
    double ip_tail;
    int nbf; bfdet_t bf[2];        /* backflow determinants (after the pair terms) */
    /* walker layout (offsets into one walker's double record) */
    long W, o_pos, o_dist, o_grad, o_lap, o_scal, o_lpc, o_gc, o_lc;
    long o_pgrad, o_plap, o_pgc, o_plc;   /* phase planes (complex determinant) */
    long o_A[MAXB], o_D[MAXB], o_Dg[MAXB], o_Dl[MAXB], o_rabs[MAXB], o_bs[MAXB];
    long o_rho[MAXT], o_pc[MAXT];
    int ncomp;
    double* blob;
} sys_t;

/* scalars of a walker record, at o_scal */
enum { S_LOGPSI, S_EL, S_WEIGHT, S_EPREV, S_RRP, S_RRA, S_AGE, S_ID, S_PARENT, S_ERR, S_ELI,
       S_NSCAL };

/* blob reader */
typedef struct { const double* p; long n, i; int bad; } rd_t;
static double rd(rd_t* r) {
    if (r->i >= r->n) { r->bad = 1; return 0.0; }
    return r->p[r->i++];
}
static const double* rdv(rd_t* r, long n) {
    if (n < 0 || r->i + n > r->n) { r->bad = 1; return r->p; }
    const double* v = r->p + r->i;
    r->i += n;
    return v;
}
static void rd_spline(rd_t* r, spline_t* s) {
    s->r_cut = rd(r);
    s->inv_delta = rd(r);
    s->n_knots = (int)rd(r);
    s->scaled = rdv(r, 3L * s->n_knots);
}

static void gauss_reduce_2d(double* a) {
    for (int guard = 0; guard < 64; ++guard) {
        const double n0 = a[0] * a[0] + a[1] * a[1];
        const double n1 = a[2] * a[2] + a[3] * a[3];
        if (n1 < n0) {
            double t = a[0]; a[0] = a[2]; a[2] = t;
            t = a[1]; a[1] = a[3]; a[3] = t;
            continue;
        }
        if (n0 == 0.0) return;
        const double mu = nearbyint((a[0] * a[2] + a[1] * a[3]) / n0);
        if (mu == 0.0) return;
        a[2] -= mu * a[0];
        a[3] -= mu * a[1];
    }
}

/* Cell from the (already reduced) lattice vectors: simulation_cell.cpp:160-270. */
static void cell_finalize(sys_t* s) {
    const int dim = s->dim;
    int ortho = 1;
    for (int i = 0; i < dim; ++i)
        for (int d = 0; d < dim; ++d)
            if (i != d && s->a[i * dim + d] != 0.0) ortho = 0;
    s->ortho = ortho;
    if (!ortho && dim == 2) gauss_reduce_2d(s->a);
    if (dim == 2) {
        const double det = s->a[0] * s->a[3] - s->a[1] * s->a[2];
        const double inv_det = 1.0 / det;
        s->ainv[0] = s->a[3] * inv_det;
        s->ainv[1] = -s->a[2] * inv_det;
        s->ainv[2] = -s->a[1] * inv_det;
        s->ainv[3] = s->a[0] * inv_det;
    } else if (dim == 1) {
        s->ainv[0] = 1.0 / s->a[0];
    } else {
        for (int d = 0; d < 3; ++d) s->ainv[d * 3 + d] = 1.0 / s->a[d * 3 + d];
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < dim * dim; ++k) s->recip[k] = two_pi * s->ainv[k];
    if (ortho)
        for (int d = 0; d < dim; ++d) {
            s->box[d] = fabs(s->a[d * dim + d]);
            s->inv_box[d] = 1.0 / s->box[d];
        }
    s->ncand = 1;
    for (int d = 0; d < 3; ++d) s->cand[d] = 0.0;
    if (!ortho && dim == 2) {
        for (int n0 = -1; n0 <= 1; ++n0)
            for (int n1 = -1; n1 <= 1; ++n1) {
                if (n0 == 0 && n1 == 0) continue;
                const double n[2] = {(double)n0, (double)n1};
                for (int d = 0; d < 2; ++d) {
                    double acc = 0.0;
                    for (int i = 0; i < 2; ++i) acc += n[i] * s->a[i * 2 + d];
                    s->cand[s->ncand * 3 + d] = acc;
                }
                s->ncand++;
            }
    }
}

/* Minimum image of a 2-D or orthorhombic displacement, in place. */
static void min_image(const sys_t* s, double* del) {
    if (!s->periodic) return;
    if (s->ortho) {
        for (int d = 0; d < s->dim; ++d) del[d] = del[d] - s->box[d] * nearbyint(del[d] * s->inv_box[d]);
        return;
    }
    double x0 = del[0], x1 = del[1];
    double s0 = 0.0;
    s0 += s->ainv[0] * x0;
    s0 += s->ainv[1] * x1;
    double s1 = 0.0;
    s1 += s->ainv[2] * x0;
    s1 += s->ainv[3] * x1;
    const double f0 = nearbyint(s0), f1 = nearbyint(s1);
    double t0 = 0.0;
    t0 += f0 * s->a[0];
    t0 += f1 * s->a[2];
    double t1 = 0.0;
    t1 += f0 * s->a[1];
    t1 += f1 * s->a[3];
    x0 -= t0;
    x1 -= t1;
    double b0 = x0, b1 = x1, best2 = 0.0;
    best2 += x0 * x0;
    best2 += x1 * x1;
    for (int c = 1; c < 9; ++c) {
        const double y0 = x0 + s->cand[c * 3 + 0];
        double r2 = 0.0;
        r2 += y0 * y0;
        const double y1 = x1 + s->cand[c * 3 + 1];
        r2 += y1 * y1;
        const double take = (r2 < best2) ? 1.0 : 0.0;
        best2 += take * (r2 - best2);
        b0 += take * (y0 - b0);
        b1 += take * (y1 - b1);
    }
    del[0] = b0;
    del[1] = b1;
}

static void wrap(const sys_t* s, double* r) {
    if (!s->periodic) return;
    if (s->ortho) {
        for (int d = 0; d < s->dim; ++d) r[d] -= s->box[d] * nearbyint(r[d] * s->inv_box[d]);
        return;
    }
    double f[3];
    for (int i = 0; i < s->dim; ++i) {
        double acc = 0.0;
        for (int d = 0; d < s->dim; ++d) acc += s->ainv[i * s->dim + d] * r[d];
        f[i] = nearbyint(acc);
    }
    for (int d = 0; d < s->dim; ++d) {
        double acc = 0.0;
        for (int i = 0; i < s->dim; ++i) acc += f[i] * s->a[i * s->dim + d];
        r[d] -= acc;
    }
}

/* Folded displacement xi - xj and its length, the way update_batch forms it. */
static double fold_dist(const sys_t* s, const double* xi, const double* xj, double* del) {
    for (int d = 0; d < s->dim; ++d) del[d] = xi[d] - xj[d];
    min_image(s, del);
    double r2 = 0.0;
    for (int d = 0; d < s->dim; ++d) r2 += del[d] * del[d];
    return sqrt(r2);
}

/* e^x K0(x), e^x K1(x) for x > 0 (numerics/scaled_bessel_k01.h): the ascending
 * series (DLMF 10.31.1-2) for x <= 2, else the Chebyshev series in 4/x - 1 of
 * sqrt(x) e^x K_nu(x), summed by Clenshaw's recurrence. */
static void k01e(const double* cheb, double x, double* k0e, double* k1e) {
    if (x <= 2.0) {
        const double euler_gamma = 0.57721566490153286060651209008240243;
        const double y = 0.25 * x * x;
        double term0 = 1.0, term1 = 1.0, harmonic = 0.0;
        double i0 = 0.0, s0 = 0.0, i1 = 0.0, s1 = 0.0;
        for (int k = 0; k < 15; ++k) {
            if (k > 0) {
                term0 *= y / ((double)k * k);
                term1 *= y / ((double)k * (k + 1));
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
        *k0e = ex * k0;
        *k1e = ex * k1;
        return;
    }
    const double xi = 4.0 / x - 1.0, two_xi = 2.0 * xi;
    double b0 = 0.0, b0p = 0.0, b1 = 0.0, b1p = 0.0;
    for (int k = 23; k >= 1; --k) {
        const double t0 = two_xi * b0 - b0p + cheb[k];
        const double t1 = two_xi * b1 - b1p + cheb[24 + k];
        b0p = b0; b0 = t0;
        b1p = b1; b1 = t1;
    }
    const double isx = 1.0 / sqrt(x);
    *k0e = (xi * b0 - b0p + cheb[0]) * isx;
    *k1e = (xi * b1 - b1p + cheb[24]) * isx;
}

/* u0 = ln K0(kappa r^-s) and its r-derivatives (ZeroEnergyFunction::
 * zero_energy_solution). */
static void ze_solution(const term_t* T, double r, double* u0, double* du0, double* d2u0) {
    const double x = T->ze_kappa * pow(r, -T->ze_s);
    double k0e, k1e;
    k01e(T->ze_cheb, x, &k0e, &k1e);
    const double q = k1e / k0e;
    const double sx = T->ze_s * x;
    *u0 = log(k0e) - x;
    *du0 = sx * q / r;
    *d2u0 = sx / (r * r) * (sx * (1.0 - q) * (1.0 + q) - q);
}

/*
 * Blob layout (all float64; integers stored exactly):
 *   dim, np, periodic, vectors[dim*dim]
 *   ngroups; per group: first, last, charge, inv_mass[dim]
 *   nblocks; per block: first, last, type,
 *            type 0: k[n*dim], is_sin[n];  type 1: centers[n*dim], alphas[n];
 *            type 2: q[n*dim] (twisted plane waves; every block then type 2)
 *   nterms; per term: kind,
 *     kind 0 (Padé): npairs(=1), pair[4], nnum, nden, coef[nnum+nden], image,
 *                    image != 0: spline(r_cut, inv_delta, n_knots, scaled[3 n]),
 *                                u_inf, nk, n1[nk], n2[nk], kx[nk], ky[nk], w[nk]
 *     kind 1 (Drummond): npairs, pairs[4*npairs], C, gamma, L, ncoef, coef[ncoef]
 *     kind 2 (zero-energy): npairs(=1), pair[4], b, exponent, R_m, r_c, cheb[48]
 *   ewald; if ewald: spline, r_cut, inv_eps, constant, nk, n1, n2, w
 *   ncoul; per term: pair[4], coef (q_a q_b / eps)
 *   nip; per term: pair[4], strength, exponent, tail   (optional: absent = 0)
 *   nbf; per backflow determinant: first, last, type, type 0: k, is_sin;
 *        type 1: centers, alphas; nch; per channel: source_first, source_last,
 *        C, L, ncoef, coeffs[ncoef]   (optional)
 */
static int blob_read(sys_t* s, const double* blob, long n) {
    rd_t r = {blob, n, 0, 0};
    s->dim = (int)rd(&r);
    s->np = (int)rd(&r);
    s->periodic = (int)rd(&r);
    if (s->dim < 1 || s->dim > 3 || s->np < 1) return -1;
    if (s->periodic) {
        const double* v = rdv(&r, s->dim * s->dim);
        for (int k = 0; k < s->dim * s->dim; ++k) s->a[k] = v[k];
        cell_finalize(s);
    }
    s->inv_mass = calloc((size_t)s->np * s->dim, sizeof(double));
    s->charge = calloc((size_t)s->np, sizeof(double));
    s->ngroups = (int)rd(&r);
    if (s->ngroups > MAXG) return -2;
    for (int g = 0; g < s->ngroups; ++g) {
        s->gfirst[g] = (int)rd(&r);
        s->glast[g] = (int)rd(&r);
        s->gcharge[g] = rd(&r);
        const double* im = rdv(&r, s->dim);
        for (int i = s->gfirst[g]; i < s->glast[g] && i < s->np; ++i) {
            s->charge[i] = s->gcharge[g];
            for (int d = 0; d < s->dim; ++d) s->inv_mass[i * s->dim + d] = im[d];
        }
    }
    s->nblocks = (int)rd(&r);
    if (s->nblocks > MAXB) return -3;
    for (int b = 0; b < s->nblocks; ++b) {
        block_t* B = &s->blocks[b];
        B->first = (int)rd(&r);
        B->last = (int)rd(&r);
        B->type = (int)rd(&r);
        const int nb = B->last - B->first;
        if (B->type == 0) {
            B->k = rdv(&r, (long)nb * s->dim);
            B->is_sin = rdv(&r, nb);
        } else if (B->type == 2) {
            B->k = rdv(&r, (long)nb * s->dim);
            s->cplx = 1;
        } else {
            B->centers = rdv(&r, (long)nb * s->dim);
            B->alphas = rdv(&r, nb);
        }
    }
    s->nterms = (int)rd(&r);
    if (s->nterms > MAXT) return -4;
    for (int t = 0; t < s->nterms; ++t) {
        term_t* T = &s->terms[t];
        memset(T, 0, sizeof *T);
        T->kind = (int)rd(&r);
        T->npairs = (int)rd(&r);
        if (T->npairs > MAXPAIR || T->npairs < 1) return -5;
        for (int q = 0; q < T->npairs; ++q)
            for (int k = 0; k < 4; ++k) T->pairs[q][k] = (int)rd(&r);
        if (T->kind == 0) {
            T->nnum = (int)rd(&r);
            T->nden = (int)rd(&r);
            for (int k = 0; k < T->nnum + T->nden && k < 16; ++k) T->coef[k] = rd(&r);
            T->image = (int)rd(&r);
            if (T->image) {
                rd_spline(&r, &T->sp);
                T->u_inf = rd(&r);
                T->nk = (int)rd(&r);
                T->n1 = rdv(&r, T->nk);
                T->n2 = rdv(&r, T->nk);
                T->kx = rdv(&r, T->nk);
                T->ky = rdv(&r, T->nk);
                T->w = rdv(&r, T->nk);
                T->kx2 = malloc(sizeof(double) * (T->nk + 1));
                T->ky2 = malloc(sizeof(double) * (T->nk + 1));
                for (int k = 0; k < T->nk; ++k) {
                    T->kx2[k] = T->kx[k] * T->kx[k];
                    T->ky2[k] = T->ky[k] * T->ky[k];
                    if (abs((int)T->n1[k]) > T->m1) T->m1 = abs((int)T->n1[k]);
                    if (abs((int)T->n2[k]) > T->m2) T->m2 = abs((int)T->n2[k]);
                }
                const int same = T->pairs[0][0] == T->pairs[0][2] && T->pairs[0][1] == T->pairs[0][3];
                T->n_cached = (T->pairs[0][1] - T->pairs[0][0]) +
                              (same ? 0 : T->pairs[0][3] - T->pairs[0][2]);
            }
        } else if (T->kind == 2) {
            const double b = rd(&r), p = rd(&r);
            T->ze_rm = rd(&r);
            T->ze_rc = rd(&r);
            T->ze_cheb = rdv(&r, 48);
            T->ze_s = 0.5 * (p - 2.0);
            T->ze_kappa = sqrt(b) / T->ze_s;
            /* matching at R_m: u, u' continuous, u(r_c) = 0 */
            double u0, du0, d2u0;
            ze_solution(T, T->ze_rm, &u0, &du0, &d2u0);
            const double c = 2.0 * T->ze_rc - T->ze_rm;
            const double h = 1.0 / (T->ze_rm * T->ze_rm) - 1.0 / (c * c);
            T->ze_c3 = du0 / h;
            T->ze_logc2 = 2.0 * T->ze_c3 / T->ze_rc;
            T->ze_logc1 = T->ze_logc2 - T->ze_c3 / T->ze_rm - T->ze_c3 / c - u0;
        } else {
            T->C = (int)rd(&r);
            T->gamma = rd(&r);
            T->L = rd(&r);
            T->ncoef = (int)rd(&r);
            for (int k = 0; k < T->ncoef && k < 16; ++k) T->dc[k] = rd(&r);
            double ipw = 1.0;
            for (int i = 0; i < T->C; ++i) ipw *= -T->L;
            T->alpha1 = T->gamma / ipw + (T->ncoef ? T->dc[0] : 0.0) * (double)T->C / T->L;
        }
    }
    s->ewald = (int)rd(&r);
    if (s->ewald) {
        rd_spline(&r, &s->esp);
        s->e_rcut = rd(&r);
        s->e_inv_eps = rd(&r);
        s->e_const = rd(&r);
        s->enk = (int)rd(&r);
        s->en1 = rdv(&r, s->enk);
        s->en2 = rdv(&r, s->enk);
        s->ew = rdv(&r, s->enk);
        s->en1max = s->en2max = 0;
        for (int k = 0; k < s->enk; ++k) {
            if (abs((int)s->en1[k]) > s->en1max) s->en1max = abs((int)s->en1[k]);
            if (abs((int)s->en2[k]) > s->en2max) s->en2max = abs((int)s->en2[k]);
        }
    }
    s->ncoul = (int)rd(&r);
    if (s->ncoul > MAXC) return -6;
    for (int c = 0; c < s->ncoul; ++c) {
        for (int k = 0; k < 4; ++k) s->coul[c][k] = (int)rd(&r);
        s->coul_coef[c] = rd(&r);
    }
    s->nip = 0;
    s->ip_tail = 0.0;
    if (r.i < r.n) {
        s->nip = (int)rd(&r);
        if (s->nip > MAXC) return -8;
        for (int c = 0; c < s->nip; ++c) {
            for (int k = 0; k < 4; ++k) s->ip[c][k] = (int)rd(&r);
            s->ip_c[c] = rd(&r);
            s->ip_p[c] = rd(&r);
            s->ip_tail += rd(&r);
            const double rp = nearbyint(s->ip_p[c]);
            s->ip_pint[c] = (rp == s->ip_p[c] && rp <= 16.0) ? (int)rp : 0;
        }
    }
    s->nbf = 0;
    if (r.i < r.n) {
        s->nbf = (int)rd(&r);
        if (s->nbf > 2) return -9;
        for (int d = 0; d < s->nbf; ++d) {
            bfdet_t* D = &s->bf[d];
            D->first = (int)rd(&r);
            D->last = (int)rd(&r);
            D->type = (int)rd(&r);
            const int n = D->last - D->first;
            if (n < 1 || n > 64) return -10;
            if (D->type == 0) {
                D->k = rdv(&r, (long)n * s->dim);
                D->is_sin = rdv(&r, n);
            } else {
                D->centers = rdv(&r, (long)n * s->dim);
                D->alphas = rdv(&r, n);
            }
            D->nch = (int)rd(&r);
            if (D->nch > 4 || (long)n * s->np > BF_MAXE || s->dim != 2) return -11;
            for (int c = 0; c < D->nch; ++c) {
                bfch_t* C = &D->ch[c];
                C->sf = (int)rd(&r);
                C->sl = (int)rd(&r);
                C->C = (int)rd(&r);
                C->L = rd(&r);
                C->nc = (int)rd(&r);
                if (C->nc > 16 || C->nc < 1) return -12;
                for (int q = 0; q < C->nc; ++q) C->c[q] = rd(&r);
            }
        }
    }
    return r.bad ? -7 : 0;
}

static void layout(sys_t* s) {
    const long np = s->np, dim = s->dim;
    long o = 0;
    s->o_pos = o; o += np * dim;
    s->o_dist = o; o += np * np;
    s->o_grad = o; o += np * dim;
    s->o_lap = o; o += np * dim;
    s->o_scal = o; o += S_NSCAL;
    s->ncomp = (s->nblocks ? 1 : 0) + s->nterms + s->nbf;
    s->o_lpc = o; o += s->ncomp;
    s->o_gc = o; o += s->ncomp * np * dim;
    s->o_lc = o; o += s->ncomp * np * dim;
    s->o_pgrad = o; o += s->cplx ? np * dim : 0;
    s->o_plap = o; o += s->cplx ? np * dim : 0;
    s->o_pgc = o; o += s->cplx ? np * dim : 0;
    s->o_plc = o; o += s->cplx ? np * dim : 0;
    for (int b = 0; b < s->nblocks; ++b) {
        const long N = s->blocks[b].last - s->blocks[b].first;
        s->o_A[b] = o; o += (s->cplx ? 2 : 1) * N * N;
        s->o_D[b] = o; o += N * N;
        s->o_Dg[b] = o; o += N * N * dim;
        s->o_Dl[b] = o; o += N * N * dim;
        s->o_rabs[b] = o; o += N;
        s->o_bs[b] = o; o += 3;   /* block log, updates, condition */
    }
    for (int t = 0; t < s->nterms; ++t) {
        const term_t* T = &s->terms[t];
        s->o_rho[t] = o; o += T->image ? 4L * T->nk : 0;
        s->o_pc[t] = o; o += T->image ? 2L * T->nk * T->n_cached : 0;
    }
    for (int d = 0; d < s->nbf; ++d) {
        bfdet_t* D = &s->bf[d];
        const long N = D->last - D->first;
        D->o_x = o; o += N * dim;
        D->o_A = o; o += N * N;
        D->o_F = o; o += N * dim;
        D->o_ls = o; o += 2;
    }
    s->W = o;
}

void* o_sys_new(const double* blob, long n) {
    zig_build();
    sys_t* s = calloc(1, sizeof(sys_t));
    s->blob = malloc(sizeof(double) * (size_t)n);
    memcpy(s->blob, blob, sizeof(double) * (size_t)n);
    if (blob_read(s, s->blob, n) != 0) {
        free(s->blob);
        free(s);
        return NULL;
    }
    layout(s);
    return s;
}

void o_sys_free(void* p) {
    sys_t* s = p;
    if (!s) return;
    for (int t = 0; t < s->nterms; ++t) {
        free(s->terms[t].kx2);
        free(s->terms[t].ky2);
    }
    free(s->inv_mass);
    free(s->charge);
    free(s->blob);
    free(s);
}

/* Offsets: W, pos, dist, grad, lap, scalars, lpc, gc, lc. */
void o_layout(void* p, long* out) {
    const sys_t* s = p;
    out[0] = s->W; out[1] = s->o_pos; out[2] = s->o_dist; out[3] = s->o_grad;
    out[4] = s->o_lap; out[5] = s->o_scal; out[6] = s->o_lpc; out[7] = s->o_gc;
    out[8] = s->o_lc; out[9] = s->ncomp; out[10] = s->cplx ? s->o_pgrad : -1;
    out[11] = s->cplx ? s->o_plap : -1;
}

/* ───────────────────────── radial functions ─────────────────────────── */

static void spline_eval3(const spline_t* sp, double r, double* f, double* df, double* d2f) {
    if (r >= sp->r_cut) { *f = *df = *d2f = 0.0; return; }
    const double t = r * sp->inv_delta;
    int i = (int)t;
    if (i > sp->n_knots - 2) i = sp->n_knots - 2;
    const double x = t - i, y = 1.0 - x;
    const double* a = sp->scaled + 3 * i;
    const double* b = a + 3;
    const double x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
    const double y2 = y * y, y3 = y2 * y, y4 = y3 * y, y5 = y4 * y;
    const double p0 = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
    const double p1 = x - 6.0 * x3 + 8.0 * x4 - 3.0 * x5;
    const double p2 = 0.5 * x2 - 1.5 * x3 + 1.5 * x4 - 0.5 * x5;
    const double q0 = 1.0 - 10.0 * y3 + 15.0 * y4 - 6.0 * y5;
    const double q1 = y - 6.0 * y3 + 8.0 * y4 - 3.0 * y5;
    const double q2 = 0.5 * y2 - 1.5 * y3 + 1.5 * y4 - 0.5 * y5;
    const double dp0 = -30.0 * x2 + 60.0 * x3 - 30.0 * x4;
    const double dp1 = 1.0 - 18.0 * x2 + 32.0 * x3 - 15.0 * x4;
    const double dp2 = x - 4.5 * x2 + 6.0 * x3 - 2.5 * x4;
    const double dq0 = -30.0 * y2 + 60.0 * y3 - 30.0 * y4;
    const double dq1 = 1.0 - 18.0 * y2 + 32.0 * y3 - 15.0 * y4;
    const double dq2 = y - 4.5 * y2 + 6.0 * y3 - 2.5 * y4;
    const double ddp0 = -60.0 * x + 180.0 * x2 - 120.0 * x3;
    const double ddp1 = -36.0 * x + 96.0 * x2 - 60.0 * x3;
    const double ddp2 = 1.0 - 9.0 * x + 18.0 * x2 - 10.0 * x3;
    const double ddq0 = -60.0 * y + 180.0 * y2 - 120.0 * y3;
    const double ddq1 = -36.0 * y + 96.0 * y2 - 60.0 * y3;
    const double ddq2 = 1.0 - 9.0 * y + 18.0 * y2 - 10.0 * y3;
    *f = a[0] * p0 + a[1] * p1 + a[2] * p2 + b[0] * q0 - b[1] * q1 + b[2] * q2;
    *df = sp->inv_delta * (a[0] * dp0 + a[1] * dp1 + a[2] * dp2 - (b[0] * dq0 - b[1] * dq1 + b[2] * dq2));
    *d2f = sp->inv_delta * sp->inv_delta *
           (a[0] * ddp0 + a[1] * ddp1 + a[2] * ddp2 + b[0] * ddq0 - b[1] * ddq1 + b[2] * ddq2);
}

static double spline_eval1(const spline_t* sp, double r) {
    if (r >= sp->r_cut) return 0.0;
    const double t = r * sp->inv_delta;
    int i = (int)t;
    if (i > sp->n_knots - 2) i = sp->n_knots - 2;
    const double x = t - i, y = 1.0 - x;
    const double* a = sp->scaled + 3 * i;
    const double* b = a + 3;
    const double x2 = x * x, x3 = x2 * x, x4 = x3 * x, x5 = x4 * x;
    const double y2 = y * y, y3 = y2 * y, y4 = y3 * y, y5 = y4 * y;
    const double p0 = 1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5;
    const double p1 = x - 6.0 * x3 + 8.0 * x4 - 3.0 * x5;
    const double p2 = 0.5 * x2 - 1.5 * x3 + 1.5 * x4 - 0.5 * x5;
    const double q0 = 1.0 - 10.0 * y3 + 15.0 * y4 - 6.0 * y5;
    const double q1 = y - 6.0 * y3 + 8.0 * y4 - 3.0 * y5;
    const double q2 = 0.5 * y2 - 1.5 * y3 + 1.5 * y4 - 0.5 * y5;
    return a[0] * p0 + a[1] * p1 + a[2] * p2 + b[0] * q0 - b[1] * q1 + b[2] * q2;
}

static void poly_acc(const double* c, int n, double r, double* v, double* dv, double* d2v) {
    double r_km1 = 1.0, r_km2 = 0.0;
    for (int i = 0; i < n; ++i) {
        const int k = i + 1;
        *v += c[i] * r_km1 * r;
        *dv += c[i] * k * r_km1;
        *d2v += c[i] * k * (k - 1) * r_km2;
        r_km2 = r_km1;
        r_km1 *= r;
    }
}

/* u, u', u'' of term T at r (the short-range part when image-summed). */
static void radial(const term_t* T, double r, double* u, double* du, double* d2u) {
    if (T->kind == 0) {
        double p = 0.0, dp = 0.0, d2p = 0.0;
        poly_acc(T->coef, T->nnum, r, &p, &dp, &d2p);
        double q = 1.0, dq = 0.0, d2q = 0.0;
        poly_acc(T->coef + T->nnum, T->nden, r, &q, &dq, &d2q);
        const double inv_q = 1.0 / q;
        *u = p * inv_q;
        *du = (dp * q - p * dq) * inv_q * inv_q;
        *d2u = (d2p - (2.0 * dp * dq - 2.0 * p * dq * dq * inv_q + p * d2q) * inv_q) * inv_q;
        if (T->image) {
            if (r >= T->sp.r_cut) { *u = *du = *d2u = 0.0; return; }
            double f, df, d2f;
            spline_eval3(&T->sp, r, &f, &df, &d2f);
            *u -= T->u_inf + f;
            *du -= df;
            *d2u -= d2f;
        }
        return;
    }
    if (T->kind == 2) {   /* ZeroEnergyFunction::evaluate */
        if (r < T->ze_rm) {
            ze_solution(T, r, u, du, d2u);
            *u += T->ze_logc1;
            return;
        }
        const double rr = r < T->ze_rc ? r : T->ze_rc;
        const double inv_r = 1.0 / rr;
        const double inv_c = 1.0 / (2.0 * T->ze_rc - rr);
        const double m = (r < T->ze_rc) ? 1.0 : 0.0;
        const double a = T->ze_c3;
        *u = m * (T->ze_logc2 - a * inv_r - a * inv_c);
        *du = m * (a * inv_r * inv_r - a * inv_c * inv_c);
        *d2u = m * (-2.0 * a * inv_r * inv_r * inv_r - 2.0 * a * inv_c * inv_c * inv_c);
        return;
    }
    /* Drummond–Towler–Needs, drummond_jastrow.cpp eval_one */
    const double t = r - T->L;
    double tCm2 = 1.0;
    for (int i = 0; i < T->C - 2; ++i) tCm2 *= t;
    const double tCm1 = tCm2 * t, tC = tCm1 * t;
    const double g = tC, dg = (double)T->C * tCm1, d2g = (double)T->C * (T->C - 1) * tCm2;
    double P = T->dc[0] + T->alpha1 * r, dP = T->alpha1, d2P = 0.0;
    double r_lm2 = 1.0, r_lm1 = r, r_l = r * r;
    for (int k = 1; k < T->ncoef; ++k) {
        const int l = k + 1;
        const double c = T->dc[k];
        P += c * r_l;
        dP += c * l * r_lm1;
        d2P += c * l * (l - 1) * r_lm2;
        r_lm2 = r_lm1;
        r_lm1 = r_l;
        r_l *= r;
    }
    const double m = (r < T->L) ? 1.0 : 0.0;
    *u = m * (g * P);
    *du = m * (dg * P + g * dP);
    *d2u = m * (d2g * P + 2.0 * dg * dP + g * d2P);
}

/* ───────────────────────── walker access ─────────────────────────────── */

#define POS(s, w) ((w) + (s)->o_pos)
#define DIST(s, w) ((w) + (s)->o_dist)
#define GRAD(s, w) ((w) + (s)->o_grad)
#define LAP(s, w) ((w) + (s)->o_lap)
#define SC(s, w) ((w) + (s)->o_scal)
#define LPC(s, w) ((w) + (s)->o_lpc)
#define GC(s, w, c) ((w) + (s)->o_gc + (long)(c) * (s)->np * (s)->dim)
#define LC(s, w, c) ((w) + (s)->o_lc + (long)(c) * (s)->np * (s)->dim)

static int term_comp(const sys_t* s, int t) { return (s->nblocks ? 1 : 0) + t; }

/* Phases e^{ik.r} of position (x, y) for term T: reciprocal_phases.h. */
static void phases(const sys_t* s, const term_t* T, double x, double y, double* c, double* sn) {
    double e1r[64], e1i[64], e2r[64], e2i[64];
    const double th1 = s->recip[0] * x + s->recip[1] * y;
    const double th2 = s->recip[2] * x + s->recip[3] * y;
    const int M[2] = {T->m1, T->m2};
    const double th[2] = {th1, th2};
    double* R[2] = {e1r, e2r};
    double* Im[2] = {e1i, e2i};
    for (int q = 0; q < 2; ++q) {
        const int m = M[q];
        double* rr = R[q] + m;
        double* ii = Im[q] + m;
        const double cc = cos(th[q]), ss = sin(th[q]);
        rr[0] = 1.0;
        ii[0] = 0.0;
        for (int n = 1; n <= m; ++n) {
            rr[n] = rr[n - 1] * cc - ii[n - 1] * ss;
            ii[n] = rr[n - 1] * ss + ii[n - 1] * cc;
            rr[-n] = rr[n];
            ii[-n] = -ii[n];
        }
    }
    const double* f1r = e1r + T->m1; const double* f1i = e1i + T->m1;
    const double* f2r = e2r + T->m2; const double* f2i = e2i + T->m2;
    for (int k = 0; k < T->nk; ++k) {
        const int a = (int)T->n1[k], b = (int)T->n2[k];
        const double ar = f1r[a], ai = f1i[a], br = f2r[b], bi = f2i[b];
        c[k] = ar * br - ai * bi;
        sn[k] = ar * bi + ai * br;
    }
}

static int t_same(const term_t* T) {
    return T->pairs[0][0] == T->pairs[0][2] && T->pairs[0][1] == T->pairs[0][3];
}
static int t_slot(const term_t* T, int i) {
    return (i >= T->pairs[0][0] && i < T->pairs[0][1]) ? i - T->pairs[0][0]
                                                         : (T->pairs[0][1] - T->pairs[0][0]) + (i - T->pairs[0][2]);
}

typedef struct { double gx, gy, lx, ly; } kterms_t;
static kterms_t kterms(const term_t* T, const double* c, const double* sn, const double* pr,
                       const double* pi, double self) {
    kterms_t t = {0, 0, 0, 0};
    for (int k = 0; k < T->nk; ++k) {
        const double g = 2.0 * T->w[k] * (c[k] * pi[k] - sn[k] * pr[k]);
        const double l = 2.0 * T->w[k] * (self - (c[k] * pr[k] + sn[k] * pi[k]));
        t.gx += T->kx[k] * g;
        t.gy += T->ky[k] * g;
        t.lx += T->kx2[k] * l;
        t.ly += T->ky2[k] * l;
    }
    return t;
}

/* ───────────────────────── orbitals ─────────────────────────────────── */

static void orbitals(const sys_t* s, const block_t* B, const double* r, double* val, double* grad,
                     double* lap) {
    const int n = B->last - B->first, dim = s->dim;
    for (int i = 0; i < n; ++i) {
        if (B->type == 0) {
            const double* ki = B->k + i * dim;
            double phase = 0.0;
            for (int d = 0; d < dim; ++d) phase += ki[d] * r[d];
            const double sn = sin(phase), c = cos(phase);
            if (B->is_sin[i] != 0.0) {
                val[i] = sn;
                for (int d = 0; d < dim; ++d) {
                    grad[i * dim + d] = ki[d] * c;
                    lap[i * dim + d] = -ki[d] * ki[d] * sn;
                }
            } else {
                val[i] = c;
                for (int d = 0; d < dim; ++d) {
                    grad[i * dim + d] = -ki[d] * sn;
                    lap[i * dim + d] = -ki[d] * ki[d] * c;
                }
            }
        } else {
            const double alpha = B->alphas[i];
            double del[3];
            for (int d = 0; d < dim; ++d) del[d] = r[d] - B->centers[i * dim + d];
            min_image(s, del);
            double r2 = 0.0;
            for (int d = 0; d < dim; ++d) r2 += del[d] * del[d];
            const double phi = exp(-alpha * r2);
            val[i] = phi;
            for (int d = 0; d < dim; ++d) {
                grad[i * dim + d] = phi * (-2.0 * alpha * del[d]);
                lap[i * dim + d] = phi * (4.0 * alpha * alpha * del[d] * del[d] - 2.0 * alpha);
            }
        }
    }
}

/* ───────────────────────── Slater determinant ───────────────────────── */

/* Pivoted Gauss-Jordan of the committed D into A; returns log|det|. */
static double gj_rebuild(int N, const double* D, double* A, int* err) {
    double m[64 * 64];
    for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) {
            m[r * N + c] = D[r * N + c];
            A[r * N + c] = r == c ? 1.0 : 0.0;
        }
    double log_det = 0.0;
    for (int k = 0; k < N; ++k) {
        int piv = k;
        for (int r = k + 1; r < N; ++r)
            if (fabs(m[r * N + k]) > fabs(m[piv * N + k])) piv = r;
        const double diag = m[piv * N + k];
        if (diag == 0.0 || !isfinite(diag)) { *err = 1; return 0.0; }
        log_det += log(fabs(diag));
        if (piv != k)
            for (int c = 0; c < N; ++c) {
                double t = m[k * N + c]; m[k * N + c] = m[piv * N + c]; m[piv * N + c] = t;
                t = A[k * N + c]; A[k * N + c] = A[piv * N + c]; A[piv * N + c] = t;
            }
        for (int c = 0; c < N; ++c) {
            m[k * N + c] /= diag;
            A[k * N + c] /= diag;
        }
        for (int r = 0; r < N; ++r) {
            if (r == k) continue;
            const double f = m[r * N + k];
            for (int c = 0; c < N; ++c) {
                m[r * N + c] -= f * m[k * N + c];
                A[r * N + c] -= f * A[k * N + c];
            }
        }
    }
    return log_det;
}

static int block_of(const sys_t* s, int p) {
    for (int b = 0; b < s->nblocks; ++b)
        if (p >= s->blocks[b].first && p < s->blocks[b].last) return b;
    return -1;
}

static void slater_evaluate(const sys_t* s, double* w) {
    const int dim = s->dim, np = s->np;
    double* gc = GC(s, w, 0);
    double* lc = LC(s, w, 0);
    LPC(s, w)[0] = 0.0;
    memset(gc, 0, sizeof(double) * np * dim);
    memset(lc, 0, sizeof(double) * np * dim);
    for (int b = 0; b < s->nblocks; ++b) {
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first;
        double* D = w + s->o_D[b];
        double* Dg = w + s->o_Dg[b];
        double* Dl = w + s->o_Dl[b];
        double* A = w + s->o_A[b];
        double* rabs = w + s->o_rabs[b];
        double* bs = w + s->o_bs[b];
        for (int kr = 0; kr < N; ++kr)
            orbitals(s, B, POS(s, w) + (B->first + kr) * dim, D + kr * N, Dg + kr * N * dim,
                     Dl + kr * N * dim);
        for (int kr = 0; kr < N; ++kr) {
            double sum = 0.0;
            for (int i = 0; i < N; ++i) sum += fabs(D[kr * N + i]);
            rabs[kr] = sum;
        }
        int err = 0;
        const double ld = gj_rebuild(N, D, A, &err);
        if (err) SC(s, w)[S_ERR] = 1.0;
        bs[0] = ld;
        bs[1] = 0.0;
        double nd = 0.0, na = 0.0;
        for (int a = 0; a < N; ++a) {
            double rd_ = 0.0, ra = 0.0;
            for (int c = 0; c < N; ++c) {
                rd_ += fabs(D[a * N + c]);
                ra += fabs(A[a * N + c]);
            }
            if (rd_ > nd) nd = rd_;
            if (ra > na) na = ra;
        }
        bs[2] = nd * na;
        LPC(s, w)[0] += ld;
        for (int kr = 0; kr < N; ++kr) {
            const int part = B->first + kr;
            for (int d = 0; d < dim; ++d) {
                double G = 0.0, Lraw = 0.0;
                for (int m = 0; m < N; ++m) {
                    const double a = A[m * N + kr];
                    G += a * Dg[(kr * N + m) * dim + d];
                    Lraw += a * Dl[(kr * N + m) * dim + d];
                }
                gc[part * dim + d] += G;
                lc[part * dim + d] += Lraw - G * G;
            }
        }
    }
}

/* Refresh particle p's Slater gradient/Laplacian into the totals
 * (slater_determinant.cpp:862-893). */
static void slater_refresh(const sys_t* s, double* w, int p) {
    const int b = block_of(s, p);
    if (b < 0 || s->cplx) return;   /* the complex determinant is eager */
    const block_t* B = &s->blocks[b];
    const int N = B->last - B->first, kr = p - B->first, dim = s->dim;
    const double* A = w + s->o_A[b];
    const double* Dg = w + s->o_Dg[b];
    const double* Dl = w + s->o_Dl[b];
    double* gc = GC(s, w, 0);
    double* lc = LC(s, w, 0);
    for (int d = 0; d < dim; ++d) {
        double grad = 0.0, lap = 0.0;
        for (int m = 0; m < N; ++m) {
            const double a = A[m * N + kr];
            grad += a * Dg[(kr * N + m) * dim + d];
            lap += a * Dl[(kr * N + m) * dim + d];
        }
        lap -= grad * grad;
        const int j = p * dim + d;
        if (grad != gc[j]) GRAD(s, w)[j] = (GRAD(s, w)[j] - gc[j]) + grad;
        if (lap != lc[j]) LAP(s, w)[j] = (LAP(s, w)[j] - lc[j]) + lap;
        gc[j] = grad;
        lc[j] = lap;
    }
}

/* ───────────────────────── complex Slater determinant ─────────────────
 * complex_slater_determinant.cpp: twisted plane waves φ_i = e^{i q_i·r}
 * (complex_orbital_set.h TwistedPlaneWaveOrbitalSet), complex inverse per
 * block stored as re[N²] then im[N²], A[m][c] = (D⁻¹)_{m,c}; ln|det| per
 * block; the modulus part of ∇ln ψ, ∂²ln ψ in the component planes and the
 * phase part in the phase planes.  Eager: every accepted move re-inverts the
 * block and recomputes all its particles' derivatives (as the reference). */

typedef double complex zc;

static zc corb(const block_t* B, int i, int dim, const double* r) {
    const double* q = B->k + i * dim;
    double arg = 0.0;
    for (int d = 0; d < dim; ++d) arg += q[d] * r[d];
    return CMPLX(cos(arg), sin(arg));
}

/* Complex Gauss-Jordan inverse of M (rows kr) into Ar/Ai; ln|det|. */
static double cgj(int N, const zc* M0, double* Ar, double* Ai, int* err) {
    zc m[64 * 64], a[64 * 64];
    for (int r = 0; r < N; ++r)
        for (int c = 0; c < N; ++c) {
            m[r * N + c] = M0[r * N + c];
            a[r * N + c] = r == c ? 1.0 : 0.0;
        }
    double log_det = 0.0;
    for (int k = 0; k < N; ++k) {
        int piv = k;
        for (int r = k + 1; r < N; ++r)
            if (cabs(m[r * N + k]) > cabs(m[piv * N + k])) piv = r;
        const zc diag = m[piv * N + k];
        if (cabs(diag) == 0.0 || !isfinite(creal(diag)) || !isfinite(cimag(diag))) { *err = 1; return 0.0; }
        log_det += log(cabs(diag));
        if (piv != k)
            for (int c = 0; c < N; ++c) {
                zc t = m[k * N + c]; m[k * N + c] = m[piv * N + c]; m[piv * N + c] = t;
                t = a[k * N + c]; a[k * N + c] = a[piv * N + c]; a[piv * N + c] = t;
            }
        const zc inv = 1.0 / diag;
        for (int c = 0; c < N; ++c) {
            m[k * N + c] *= inv;
            a[k * N + c] *= inv;
        }
        for (int r = 0; r < N; ++r) {
            if (r == k) continue;
            const zc f = m[r * N + k];
            for (int c = 0; c < N; ++c) {
                m[r * N + c] -= f * m[k * N + c];
                a[r * N + c] -= f * a[k * N + c];
            }
        }
    }
    for (int e = 0; e < N * N; ++e) {
        Ar[e] = creal(a[e]);
        Ai[e] = cimag(a[e]);
    }
    return log_det;
}

/* Rows of block b at the walker's positions (particle `moved` at `np_`). */
static void crows(const sys_t* s, const double* w, int b, int moved, const double* np_, zc* D) {
    const block_t* B = &s->blocks[b];
    const int N = B->last - B->first, dim = s->dim;
    for (int kr = 0; kr < N; ++kr) {
        const int part = B->first + kr;
        const double* r = part == moved ? np_ : POS(s, w) + part * dim;
        for (int i = 0; i < N; ++i) D[kr * N + i] = corb(B, i, dim, r);
    }
}

/* G_d = Σ_m A[m][kr] ∂_d φ_m(r), L_d = Σ_m A[m][kr] ∂²_d φ_m(r) - G_d² at r. */
static void cderivs(const sys_t* s, const double* w, int b, int kr, const double* r, zc* G, zc* L) {
    const block_t* B = &s->blocks[b];
    const int N = B->last - B->first, dim = s->dim;
    const double* Ar = w + s->o_A[b];
    const double* Ai = Ar + N * N;
    for (int d = 0; d < dim; ++d) {
        zc g = 0.0, l = 0.0;
        for (int m = 0; m < N; ++m) {
            const zc a = CMPLX(Ar[m * N + kr], Ai[m * N + kr]);
            const zc phi = corb(B, m, dim, r);
            const double qd = B->k[m * dim + d];
            g += a * (I * qd * phi);
            l += a * (-qd * qd * phi);
        }
        G[d] = g;
        L[d] = l - g * g;
    }
}

static void cslater_evaluate(const sys_t* s, double* w) {
    const int dim = s->dim, np = s->np;
    double* gc = GC(s, w, 0);
    double* lc = LC(s, w, 0);
    double* pgc = w + s->o_pgc;
    double* plc = w + s->o_plc;
    LPC(s, w)[0] = 0.0;
    memset(gc, 0, sizeof(double) * np * dim);
    memset(lc, 0, sizeof(double) * np * dim);
    memset(pgc, 0, sizeof(double) * np * dim);
    memset(plc, 0, sizeof(double) * np * dim);
    for (int b = 0; b < s->nblocks; ++b) {
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first;
        zc D[64 * 64];
        crows(s, w, b, -1, NULL, D);
        double* Ar = w + s->o_A[b];
        int err = 0;
        const double ld = cgj(N, D, Ar, Ar + N * N, &err);
        if (err) SC(s, w)[S_ERR] = 1.0;
        double* bs = w + s->o_bs[b];
        bs[0] = ld;
        bs[1] = 0.0;
        bs[2] = 0.0;
        LPC(s, w)[0] += ld;
        for (int kr = 0; kr < N; ++kr) {
            const int part = B->first + kr;
            zc G[3], L[3];
            cderivs(s, w, b, kr, POS(s, w) + part * dim, G, L);
            for (int d = 0; d < dim; ++d) {
                gc[part * dim + d] += creal(G[d]);
                lc[part * dim + d] += creal(L[d]);
                pgc[part * dim + d] += cimag(G[d]);
                plc[part * dim + d] += cimag(L[d]);
            }
        }
    }
    memcpy(w + s->o_pgrad, pgc, sizeof(double) * np * dim);
    memcpy(w + s->o_plap, plc, sizeof(double) * np * dim);
}

/* ───────────────────────── backflow determinant ──────────────────────
 * backflow_slater_determinant.cpp / backflow_transformation.cpp: rows
 * M[i][m] = φ_m(x_i), x_i = r_i + Σ_c Σ_j η_c(r_ij) r_ij (minimum image),
 * inverted per move by pivoted Gauss-Jordan; ∂_kβ ln|D| = Σ F·J and
 * ∂²_kβ ln|D| = Σ F·S + Σ_i vᵀT_i v - Σ_{ij} U_ji U_ij with the pair tables
 * B(r) = η δ + η' r̂ r̂ᵀ r and s(r) = ∂²_β[η r_α]. */

static int bf_comp(const sys_t* s, int d) { return (s->nblocks ? 1 : 0) + s->nterms + d; }

static int bf_affects(const bfdet_t* D, int k) {
    if (k >= D->first && k < D->last) return 1;
    for (int c = 0; c < D->nch; ++c)
        if (k >= D->ch[c].sf && k < D->ch[c].sl) return 1;
    return 0;
}

/* η, η', η'' of a channel at r (backflow_function.h evaluate). */
static void bf_eta(const bfch_t* C, double r, double* eta, double* e1, double* e2) {
    if (r >= C->L) { *eta = *e1 = *e2 = 0.0; return; }
    const double t = 1.0 - r / C->L;
    double tc2 = 1.0;
    for (int i = 0; i < C->C - 2; ++i) tc2 *= t;
    const double f = tc2 * t * t;
    const double fp = -(double)C->C / C->L * tc2 * t;
    const double fpp = (double)C->C * (double)(C->C - 1) / (C->L * C->L) * tc2;
    double P = 0.0, Pp = 0.0, Ppp = 0.0;
    for (int k = C->nc - 1; k >= 0; --k) {
        Ppp = Ppp * r + 2.0 * Pp;
        Pp = Pp * r + P;
        P = P * r + C->c[k];
    }
    *eta = f * P;
    *e1 = fp * P + f * Pp;
    *e2 = fpp * P + 2.0 * fp * Pp + f * Ppp;
}

/* One pair: sign η r_ij added to x; B and S (2x2) when B is given. */
static int bf_pair(const sys_t* s, const bfch_t* C, const double* ri, const double* rj, double sign,
                   double* x, double* B, double* S) {
    double del[3] = {ri[0] - rj[0], ri[1] - rj[1], 0.0};
    min_image(s, del);
    const double r = sqrt(del[0] * del[0] + del[1] * del[1]);
    if (r >= C->L) return 0;
    double eta, e1, e2;
    bf_eta(C, r, &eta, &e1, &e2);
    for (int d = 0; d < 2; ++d) x[d] += sign * eta * del[d];
    if (!B) return 1;
    const double inv_r = r > 0.0 ? 1.0 / r : 0.0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            B[a * 2 + b] = (a == b ? eta : 0.0) + e1 * del[a] * del[b] * inv_r;
            const double rb2 = del[b] * del[b] * inv_r * inv_r;
            S[a * 2 + b] = (a == b ? 2.0 * e1 * del[b] * inv_r : 0.0) +
                           del[a] * (e2 * rb2 + e1 * inv_r * (1.0 - rb2));
        }
    return 1;
}

/* pair tables of one configuration: [row * np + j] */
typedef struct { double b[BF_MAXE * 4], sx[BF_MAXE * 4]; char lk[BF_MAXE]; } bftab_t;
static bftab_t g_tab;

static void bf_clear(int np, int e) {
    g_tab.lk[e] = 0;
    (void)np;
    for (int q = 0; q < 4; ++q) g_tab.b[e * 4 + q] = g_tab.sx[e * 4 + q] = 0.0;
}

static void bf_full(const sys_t* s, const bfdet_t* D, const double* pos, double* x) {
    const int np = s->np, N = D->last - D->first;
    for (int t = 0; t < N; ++t) {
        const int P = D->first + t;
        double* xt = x + t * 2;
        xt[0] = pos[P * 2];
        xt[1] = pos[P * 2 + 1];
        for (int j = 0; j < np; ++j) bf_clear(np, t * np + j);
        for (int c = 0; c < D->nch; ++c)
            for (int j = D->ch[c].sf; j < D->ch[c].sl; ++j) {
                if (j == P) continue;
                const int e = t * np + j;
                g_tab.lk[e] = (char)bf_pair(s, &D->ch[c], pos + P * 2, pos + j * 2, 1.0, xt, g_tab.b + e * 4,
                                            g_tab.sx + e * 4);
            }
    }
}

static void bf_particle_tables(const sys_t* s, const bfdet_t* D, const double* pos, int k, double* x) {
    const int np = s->np, N = D->last - D->first;
    const int tk = (k >= D->first && k < D->last) ? k - D->first : -1;
    if (tk >= 0) {
        double* xt = x + tk * 2;
        xt[0] = pos[k * 2];
        xt[1] = pos[k * 2 + 1];
        for (int j = 0; j < np; ++j) bf_clear(np, tk * np + j);
        for (int c = 0; c < D->nch; ++c)
            for (int j = D->ch[c].sf; j < D->ch[c].sl; ++j) {
                if (j == k) continue;
                const int e = tk * np + j;
                g_tab.lk[e] = (char)bf_pair(s, &D->ch[c], pos + k * 2, pos + j * 2, 1.0, xt, g_tab.b + e * 4,
                                            g_tab.sx + e * 4);
            }
    }
    for (int t = 0; t < N; ++t) {
        const int P = D->first + t;
        if (P == k) continue;
        const int e = t * np + k;
        bf_clear(np, e);
        for (int c = 0; c < D->nch; ++c) {
            if (k < D->ch[c].sf || k >= D->ch[c].sl) continue;
            double unused[2] = {0, 0};
            g_tab.lk[e] = (char)bf_pair(s, &D->ch[c], pos + P * 2, pos + k * 2, 1.0, unused, g_tab.b + e * 4,
                                        g_tab.sx + e * 4);
        }
    }
}

static void bf_shift(const sys_t* s, const bfdet_t* D, const double* pos, int k, const double* old_r,
                     double* x) {
    for (int c = 0; c < D->nch; ++c) {
        if (k < D->ch[c].sf || k >= D->ch[c].sl) continue;
        for (int P = D->first; P < D->last; ++P) {
            if (P == k) continue;
            double* xt = x + (P - D->first) * 2;
            bf_pair(s, &D->ch[c], pos + P * 2, pos + k * 2, 1.0, xt, NULL, NULL);
            bf_pair(s, &D->ch[c], pos + P * 2, old_r, -1.0, xt, NULL, NULL);
        }
    }
}

/* orbitals with Hessians at x_i for every row: val[i*N+m], grad[(i*N+m)*2+a],
 * hess[((i*N+m)*2+a)*2+b] */
static void bf_rows(const sys_t* s, const bfdet_t* D, const double* x, double* val, double* grad,
                    double* hess) {
    const int N = D->last - D->first;
    for (int i = 0; i < N; ++i)
        for (int m = 0; m < N; ++m) {
            const double* r = x + i * 2;
            const int o = i * N + m;
            if (D->type == 0) {
                const double* km = D->k + m * 2;
                const double ph = km[0] * r[0] + km[1] * r[1];
                const double sn = sin(ph), c = cos(ph);
                const double v = D->is_sin[m] != 0.0 ? sn : c;
                const double dv = D->is_sin[m] != 0.0 ? c : -sn;
                val[o] = v;
                for (int a = 0; a < 2; ++a) {
                    grad[o * 2 + a] = km[a] * dv;
                    for (int b = 0; b < 2; ++b) hess[(o * 2 + a) * 2 + b] = -km[a] * km[b] * v;
                }
            } else {
                const double al = D->alphas[m];
                double del[3] = {r[0] - D->centers[m * 2], r[1] - D->centers[m * 2 + 1], 0.0};
                min_image(s, del);
                const double phi = exp(-al * (del[0] * del[0] + del[1] * del[1]));
                val[o] = phi;
                for (int a = 0; a < 2; ++a) {
                    grad[o * 2 + a] = -2.0 * al * del[a] * phi;
                    for (int b = 0; b < 2; ++b)
                        hess[(o * 2 + a) * 2 + b] = (4.0 * al * al * del[a] * del[b] - (a == b ? 2.0 * al : 0.0)) * phi;
                }
            }
        }
}

/* Pivoted Gauss-Jordan with log|det| and sign (m destroyed); 0 if singular. */
static int bf_invert(int n, double* m, double* a, double* log_det, double* sign) {
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) a[r * n + c] = r == c ? 1.0 : 0.0;
    *log_det = 0.0;
    *sign = 1.0;
    for (int k = 0; k < n; ++k) {
        int piv = k;
        for (int r = k + 1; r < n; ++r)
            if (fabs(m[r * n + k]) > fabs(m[piv * n + k])) piv = r;
        const double diag = m[piv * n + k];
        if (diag == 0.0 || !isfinite(diag)) return 0;
        *log_det += log(fabs(diag));
        if (diag < 0.0) *sign = -*sign;
        if (piv != k) {
            for (int c = 0; c < n; ++c) {
                double t = m[k * n + c]; m[k * n + c] = m[piv * n + c]; m[piv * n + c] = t;
                t = a[k * n + c]; a[k * n + c] = a[piv * n + c]; a[piv * n + c] = t;
            }
            *sign = -*sign;
        }
        const double inv = 1.0 / diag;
        for (int c = k + 1; c < n; ++c) m[k * n + c] *= inv;
        for (int c = 0; c < n; ++c) a[k * n + c] *= inv;
        for (int r = 0; r < n; ++r) {
            if (r == k) continue;
            const double f = m[r * n + k];
            if (f == 0.0) continue;
            for (int c = k + 1; c < n; ++c) m[r * n + c] -= f * m[k * n + c];
            for (int c = 0; c < n; ++c) a[r * n + c] -= f * a[k * n + c];
        }
    }
    return 1;
}

/* F_iα = Σ_m A[m][i] ∂_α φ_m(x_i) */
static void bf_f(int N, const double* A, const double* grad, double* F) {
    for (int i = 0; i < N; ++i)
        for (int a = 0; a < 2; ++a) {
            double acc = 0.0;
            for (int m = 0; m < N; ++m) acc += A[m * N + i] * grad[(i * N + m) * 2 + a];
            F[i * 2 + a] = acc;
        }
}

/* v = Jacobian column (k, β) over the rows; returns Σ F·S. */
static double bf_jcol(const sys_t* s, const bfdet_t* D, const double* F, int k, int beta, double* v) {
    const int np = s->np, N = D->last - D->first;
    for (int q = 0; q < N * 2; ++q) v[q] = 0.0;
    double fs = 0.0;
    const int tk = (k >= D->first && k < D->last) ? k - D->first : -1;
    if (tk >= 0) {
        double* vk = v + tk * 2;
        vk[beta] = 1.0;
        for (int j = 0; j < np; ++j) {
            const int e = tk * np + j;
            if (!g_tab.lk[e]) continue;
            for (int a = 0; a < 2; ++a) {
                vk[a] += g_tab.b[e * 4 + a * 2 + beta];
                fs += F[tk * 2 + a] * g_tab.sx[e * 4 + a * 2 + beta];
            }
        }
    }
    for (int t = 0; t < N; ++t) {
        const int e = t * np + k;
        if (t == tk || !g_tab.lk[e]) continue;
        for (int a = 0; a < 2; ++a) {
            v[t * 2 + a] = -g_tab.b[e * 4 + a * 2 + beta];
            fs += F[t * 2 + a] * g_tab.sx[e * 4 + a * 2 + beta];
        }
    }
    return fs;
}

/* ∂_k ln|D| = Σ_t F_t · ∂x_t/∂r_k */
static void bf_gradient(const sys_t* s, const bfdet_t* D, const double* F, int k, double* out) {
    const int np = s->np, N = D->last - D->first;
    out[0] = out[1] = 0.0;
    const int tk = (k >= D->first && k < D->last) ? k - D->first : -1;
    if (tk >= 0) {
        const double* Fk = F + tk * 2;
        out[0] += Fk[0];
        out[1] += Fk[1];
        for (int j = 0; j < np; ++j) {
            const int e = tk * np + j;
            if (!g_tab.lk[e]) continue;
            for (int a = 0; a < 2; ++a)
                for (int b = 0; b < 2; ++b) out[b] += Fk[a] * g_tab.b[e * 4 + a * 2 + b];
        }
    }
    for (int t = 0; t < N; ++t) {
        const int e = t * np + k;
        if (t == tk || !g_tab.lk[e]) continue;
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) out[b] -= F[t * 2 + a] * g_tab.b[e * 4 + a * 2 + b];
    }
}

/* Every particle's gradient and Laplacian from committed A, F and rows
 * (BackflowSlaterDeterminant::all_derivatives). */
static void bf_all(const sys_t* s, const bfdet_t* D, const double* A, const double* F, const double* grad,
                   const double* hess, double* g_out, double* l_out) {
    const int np = s->np, N = D->last - D->first;
    static double T[64 * 4], G[2][64 * 64], v[128], U[64 * 64];
    for (int i = 0; i < N; ++i)
        for (int ag = 0; ag < 4; ++ag) {
            double acc = 0.0;
            for (int m = 0; m < N; ++m) acc += A[m * N + i] * hess[(i * N + m) * 4 + ag];
            T[i * 4 + ag] = acc;
        }
    for (int a = 0; a < 2; ++a)
        for (int j = 0; j < N; ++j)
            for (int r = 0; r < N; ++r) {
                double acc = 0.0;
                for (int m = 0; m < N; ++m) acc += A[m * N + j] * grad[(r * N + m) * 2 + a];
                G[a][j * N + r] = acc;
            }
    for (int k = 0; k < np; ++k) {
        g_out[k * 2] = g_out[k * 2 + 1] = l_out[k * 2] = l_out[k * 2 + 1] = 0.0;
        if (!bf_affects(D, k)) continue;
        bf_gradient(s, D, F, k, g_out + k * 2);
        for (int beta = 0; beta < 2; ++beta) {
            double l = bf_jcol(s, D, F, k, beta, v);
            for (int i = 0; i < N; ++i)
                for (int a = 0; a < 2; ++a)
                    for (int g = 0; g < 2; ++g) l += v[i * 2 + a] * v[i * 2 + g] * T[i * 4 + a * 2 + g];
            for (int j = 0; j < N; ++j)
                for (int r = 0; r < N; ++r)
                    U[j * N + r] = v[r * 2] * G[0][j * N + r] + v[r * 2 + 1] * G[1][j * N + r];
            double uu = 0.0;
            for (int j = 0; j < N; ++j)
                for (int r = 0; r < N; ++r) uu += U[j * N + r] * U[r * N + j];
            l_out[k * 2 + beta] = l - uu;
        }
    }
}

static double g_bval[64 * 64], g_bgrad[64 * 64 * 2], g_bhess[64 * 64 * 4], g_bwork[64 * 64];

static void bf_evaluate(const sys_t* s, double* w, int d) {
    const bfdet_t* D = &s->bf[d];
    const int N = D->last - D->first, np = s->np, c = bf_comp(s, d);
    double* x = w + D->o_x;
    double* A = w + D->o_A;
    double* F = w + D->o_F;
    double* ls = w + D->o_ls;
    bf_full(s, D, POS(s, w), x);
    bf_rows(s, D, x, g_bval, g_bgrad, g_bhess);
    memcpy(g_bwork, g_bval, sizeof(double) * N * N);
    if (!bf_invert(N, g_bwork, A, &ls[0], &ls[1])) SC(s, w)[S_ERR] = 1.0;
    bf_f(N, A, g_bgrad, F);
    bf_all(s, D, A, F, g_bgrad, g_bhess, GC(s, w, c), LC(s, w, c));
    LPC(s, w)[c] = ls[0];
    (void)np;
}

/* refresh_walker: x rebuilt from the positions, every particle's derivatives
 * from the committed A and F, into the component and (by difference) the
 * totals. */
static void bf_refresh_all(const sys_t* s, double* w, int d) {
    const bfdet_t* D = &s->bf[d];
    const int np = s->np, c = bf_comp(s, d);
    double* x = w + D->o_x;
    bf_full(s, D, POS(s, w), x);
    bf_rows(s, D, x, g_bval, g_bgrad, g_bhess);
    static double go[2048], lo[2048];
    bf_all(s, D, w + D->o_A, w + D->o_F, g_bgrad, g_bhess, go, lo);
    double* gc = GC(s, w, c);
    double* lc = LC(s, w, c);
    for (int j = 0; j < np * 2; ++j) {
        if (go[j] != gc[j]) GRAD(s, w)[j] = (GRAD(s, w)[j] - gc[j]) + go[j];
        if (lo[j] != lc[j]) LAP(s, w)[j] = (LAP(s, w)[j] - lc[j]) + lo[j];
        gc[j] = go[j];
        lc[j] = lo[j];
    }
}

/* refresh_particle_derivatives: the gradient of p only (what a drift reads). */
static void bf_refresh_particle(const sys_t* s, double* w, int d, int p) {
    const bfdet_t* D = &s->bf[d];
    if (!bf_affects(D, p)) return;
    const int c = bf_comp(s, d);
    static double xs[128];
    bf_particle_tables(s, D, POS(s, w), p, xs);
    double g[2];
    bf_gradient(s, D, w + D->o_F, p, g);
    double* gc = GC(s, w, c);
    for (int k = 0; k < 2; ++k) {
        const int j = p * 2 + k;
        if (g[k] != gc[j]) GRAD(s, w)[j] = (GRAD(s, w)[j] - gc[j]) + g[k];
        gc[j] = g[k];
    }
}

/* ───────────────────────── move scratch ─────────────────────────────── */

typedef struct {
    double new_pos[3], pend[1024];      /* pending distances [np] */
    double new_grad[3], new_lap[3], log_ratio, phase;
    double new_pgrad[3], new_plap[3];   /* phase part (complex determinant) */
    double nval[64], ngrad[64 * 3], nlap[64 * 3];
    double pg[MAXT][3], pl[MAXT][3];    /* per-term pending grad/lap */
    double rad[MAXT][1024][6];          /* u_old, du_old, d2u_old, u_new, du_new, d2u_new */
    double pc[MAXT][512], ps[MAXT][512];/* pending phases */
    /* backflow: pending x, A, F, (log|det|, sign), p's gradient, validity */
    double bx[2][128], bA[2][64 * 64], bF[2][128], bls[2][2], bg[2][2];
    int bvalid[2], bused[2];
} move_t;

/* Does term T couple particles p and k?  Calls f for every partner of p. */
static int term_partners(const term_t* T, int p, int* out) {
    int n = 0;
    for (int q = 0; q < T->npairs; ++q) {
        const int af = T->pairs[q][0], al = T->pairs[q][1], bf = T->pairs[q][2], bl = T->pairs[q][3];
        if (af == bf && al == bl) {
            if (p < af || p >= al) continue;
            for (int k = af; k < al; ++k)
                if (k != p) out[n++] = k;
        } else if (p >= af && p < al) {
            for (int k = bf; k < bl; ++k) out[n++] = k;
        } else if (p >= bf && p < bl) {
            for (int k = af; k < al; ++k) out[n++] = k;
        }
    }
    return n;
}

static void term_evaluate(const sys_t* s, double* w, int t) {
    const term_t* T = &s->terms[t];
    const int c = term_comp(s, t), dim = s->dim, np = s->np;
    double* gc = GC(s, w, c);
    double* lc = LC(s, w, c);
    double* lpc = LPC(s, w) + c;
    *lpc = 0.0;
    memset(gc, 0, sizeof(double) * np * dim);
    memset(lc, 0, sizeof(double) * np * dim);
    const double* pos = POS(s, w);
    for (int q = 0; q < T->npairs; ++q) {
        const int af = T->pairs[q][0], al = T->pairs[q][1], bf = T->pairs[q][2], bl = T->pairs[q][3];
        const int same = af == bf && al == bl;
        for (int i = af; i < al; ++i)
            for (int j = same ? i + 1 : bf; j < (same ? al : bl); ++j) {
                double del[3];
                for (int d = 0; d < dim; ++d) del[d] = pos[i * dim + d] - pos[j * dim + d];
                min_image(s, del);
                const double r = DIST(s, w)[i * np + j];
                double u, du, d2u;
                radial(T, r, &u, &du, &d2u);
                const double invr = 1.0 / r;
                *lpc += u;
                for (int d = 0; d < dim; ++d) {
                    const double dor = del[d] * invr;
                    const double g = du * dor;
                    gc[i * dim + d] += g;
                    gc[j * dim + d] -= g;
                    const double lap_d = d2u * dor * dor + du * invr * (1.0 - dor * dor);
                    lc[i * dim + d] += lap_d;
                    lc[j * dim + d] += lap_d;
                }
            }
    }
    if (!T->image) return;
    /* k-space half (kspace_pair_sum.cpp:139-160 evaluate, :105-137 accumulate) */
    const int same = t_same(T), nk = T->nk;
    const int af = T->pairs[0][0], al = T->pairs[0][1], bf = T->pairs[0][2], bl = T->pairs[0][3];
    double* rho = w + s->o_rho[t];   /* ra_re, ra_im, rb_re, rb_im */
    double* pcache = w + s->o_pc[t]; /* [slot][cos nk | sin nk] */
    for (int g = 0; g < (same ? 1 : 2); ++g) {
        const int f0 = g == 0 ? af : bf, f1 = g == 0 ? al : bl;
        double* re = rho + (g == 0 ? 0 : 2 * nk);
        double* im = re + nk;
        for (int k = 0; k < nk; ++k) re[k] = im[k] = 0.0;
        for (int i = f0; i < f1; ++i) {
            double* cc = pcache + 2L * nk * t_slot(T, i);
            double* ss = cc + nk;
            phases(s, T, pos[i * dim], pos[i * dim + 1], cc, ss);
            for (int k = 0; k < nk; ++k) { re[k] += cc[k]; im[k] += ss[k]; }
        }
    }
    const double *ar = rho, *ai = rho + nk;
    const double *br = same ? ar : rho + 2 * nk, *bi = same ? ai : rho + 3 * nk;
    double tt = 0.0;
    if (same)
        for (int k = 0; k < nk; ++k) tt += T->w[k] * (ar[k] * ar[k] + ai[k] * ai[k]);
    else
        for (int k = 0; k < nk; ++k) tt += 2.0 * T->w[k] * (ar[k] * br[k] + ai[k] * bi[k]);
    *lpc += tt;
    for (int i = af; i < al; ++i) {
        const double* cc = pcache + 2L * nk * t_slot(T, i);
        kterms_t kt = kterms(T, cc, cc + nk, br, bi, same ? 1.0 : 0.0);
        gc[i * dim] += kt.gx; gc[i * dim + 1] += kt.gy;
        lc[i * dim] += kt.lx; lc[i * dim + 1] += kt.ly;
    }
    if (!same)
        for (int j = bf; j < bl; ++j) {
            const double* cc = pcache + 2L * nk * t_slot(T, j);
            kterms_t kt = kterms(T, cc, cc + nk, ar, ai, 0.0);
            gc[j * dim] += kt.gx; gc[j * dim + 1] += kt.gy;
            lc[j * dim] += kt.lx; lc[j * dim + 1] += kt.ly;
        }
}

/* Distances of all pairs (build_all), positions wrapped first (load_all). */
static void build_tables(const sys_t* s, double* w) {
    const int np = s->np, dim = s->dim;
    double* pos = POS(s, w);
    for (int p = 0; p < np; ++p) wrap(s, pos + p * dim);
    for (int i = 0; i < np; ++i)
        for (int j = 0; j < np; ++j) {
            double del[3];
            if (s->periodic) {
                DIST(s, w)[i * np + j] = fold_dist(s, pos + i * dim, pos + j * dim, del);
            } else {
                double r2 = 0.0;
                for (int d = 0; d < dim; ++d) {
                    const double diff = pos[i * dim + d] - pos[j * dim + d];
                    r2 += diff * diff;
                }
                DIST(s, w)[i * np + j] = sqrt(r2);
            }
        }
}

/* TrialWavefunction::evaluate_batch: totals = Σ components. */
static void psi_evaluate(const sys_t* s, double* w) {
    const int n = s->np * s->dim;
    if (s->nblocks) {
        if (s->cplx) cslater_evaluate(s, w);
        else slater_evaluate(s, w);
    }
    for (int t = 0; t < s->nterms; ++t) term_evaluate(s, w, t);
    for (int d = 0; d < s->nbf; ++d) bf_evaluate(s, w, d);
    double lp = 0.0;
    memset(GRAD(s, w), 0, sizeof(double) * n);
    memset(LAP(s, w), 0, sizeof(double) * n);
    for (int c = 0; c < s->ncomp; ++c) {
        lp += LPC(s, w)[c];
        for (int k = 0; k < n; ++k) {
            GRAD(s, w)[k] += GC(s, w, c)[k];
            LAP(s, w)[k] += LC(s, w, c)[k];
        }
    }
    SC(s, w)[S_LOGPSI] = lp;
}

/* ───────────────────────── Hamiltonian ──────────────────────────────── */

static double local_energy(const sys_t* s, const double* w) {
    const int np = s->np, dim = s->dim;
    double le = 0.0;
    /* kinetic (Kinetic::evaluate_batch; add_phase_terms for a complex ψ) */
    for (int i = 0; i < np; ++i)
        for (int d = 0; d < dim; ++d) {
            const double g = GRAD(s, w)[i * dim + d], l = LAP(s, w)[i * dim + d];
            le += -0.5 * s->inv_mass[i * dim + d] * (l + g * g);
        }
    if (s->cplx)
        for (int i = 0; i < np; ++i)
            for (int d = 0; d < dim; ++d) {
                const double pg = w[s->o_pgrad + i * dim + d];
                le += 0.5 * s->inv_mass[i * dim + d] * pg * pg;
            }
    const double* dist = DIST(s, w);
    if (s->ewald) {
        /* real space, group pairs g <= h */
        for (int g = 0; g < s->ngroups; ++g)
            for (int h = g; h < s->ngroups; ++h)
                for (int i = s->gfirst[g]; i < s->glast[g]; ++i)
                    for (int j = (g == h ? i + 1 : s->gfirst[h]); j < s->glast[h]; ++j) {
                        const double coeff = s->charge[i] * s->charge[j];
                        if (coeff == 0.0) continue;
                        const double r = dist[i * np + j];
                        const double v = s->e_inv_eps / r;
                        le += r < s->e_rcut ? coeff * (v - spline_eval1(&s->esp, r)) : 0.0;
                    }
        /* reciprocal space */
        const double* pos = POS(s, w);
        const int m1 = s->en1max, m2 = s->en2max;
        double* e1r = malloc(sizeof(double) * (m1 + 1) * np);
        double* e1i = malloc(sizeof(double) * (m1 + 1) * np);
        double* e2r = malloc(sizeof(double) * (m2 + 1) * np);
        double* e2i = malloc(sizeof(double) * (m2 + 1) * np);
        for (int q = 0; q < 2; ++q) {
            const double bx = s->recip[q * 2], by = s->recip[q * 2 + 1];
            const int nmax = q == 0 ? m1 : m2;
            double* er = q == 0 ? e1r : e2r;
            double* ei = q == 0 ? e1i : e2i;
            for (int i = 0; i < np; ++i) {
                er[i] = 1.0;
                ei[i] = 0.0;
                if (nmax < 1) continue;
                const double ph = bx * pos[i * dim] + by * pos[i * dim + 1];
                er[np + i] = cos(ph);
                ei[np + i] = sin(ph);
                for (int n = 2; n <= nmax; ++n) {
                    const double pr = er[(n - 1) * np + i], pi = ei[(n - 1) * np + i];
                    er[n * np + i] = pr * er[np + i] - pi * ei[np + i];
                    ei[n * np + i] = pr * ei[np + i] + pi * er[np + i];
                }
            }
        }
        for (int kk = 0; kk < s->enk; ++kk) {
            const int n1 = (int)s->en1[kk], n2 = (int)s->en2[kk];
            const int a2 = abs(n2);
            const double sgn = n2 < 0 ? -1.0 : 1.0;
            double rr = 0.0, ri = 0.0;
            for (int i = 0; i < np; ++i) {
                const double q = s->charge[i];
                if (q == 0.0) continue;
                const double ar = e1r[n1 * np + i], ai = e1i[n1 * np + i];
                const double br = e2r[a2 * np + i], bim = sgn * e2i[a2 * np + i];
                rr += q * (ar * br - ai * bim);
                ri += q * (ar * bim + ai * br);
            }
            le += s->ew[kk] * (rr * rr + ri * ri);
        }
        free(e1r); free(e1i); free(e2r); free(e2i);
        le += s->e_const;
    }
    for (int c = 0; c < s->ncoul; ++c) {
        const int af = s->coul[c][0], al = s->coul[c][1], bf = s->coul[c][2], bl = s->coul[c][3];
        const int same = af == bf && al == bl;
        for (int i = af; i < al; ++i)
            for (int j = same ? i + 1 : bf; j < (same ? al : bl); ++j) {
                const double r = dist[i * np + j];
                le += s->coul_coef[c] / sqrt(r * r + 0.0);
            }
    }
    /* InversePowerTerm::evaluate_potential: C r^-p at the minimum image, plus tail */
    for (int c = 0; c < s->nip; ++c) {
        const int af = s->ip[c][0], al = s->ip[c][1], bf = s->ip[c][2], bl = s->ip[c][3];
        const int same = af == bf && al == bl;
        for (int i = af; i < al; ++i)
            for (int j = same ? i + 1 : bf; j < (same ? al : bl); ++j) {
                const double r = dist[i * np + j];
                if (s->ip_pint[c] > 0) {
                    const double inv_r = 1.0 / r;
                    double inv_rp = inv_r;
                    for (int k = 1; k < s->ip_pint[c]; ++k) inv_rp *= inv_r;
                    le += s->ip_c[c] * inv_rp;
                } else {
                    le += s->ip_c[c] * pow(r, -s->ip_p[c]);
                }
            }
    }
    le += s->ip_tail;
    return le;
}

/* Imaginary part of E_L of a complex ψ: -½ Σ (1/m)(∂²φ + 2 ∂ln|ψ|·∂φ)
 * (Kinetic::add_phase_terms). */
static double local_energy_imag(const sys_t* s, const double* w) {
    if (!s->cplx) return 0.0;
    double im = 0.0;
    for (int i = 0; i < s->np; ++i)
        for (int d = 0; d < s->dim; ++d) {
            const int k = i * s->dim + d;
            im += -0.5 * s->inv_mass[k] * (w[s->o_plap + k] + 2.0 * GRAD(s, w)[k] * w[s->o_pgrad + k]);
        }
    return im;
}

/* Initialise walkers from AoS positions [w][p][d] and evaluate psi and H. */
int o_init(void* p, double* walkers, long nw, const double* pos_aos) {
    const sys_t* s = p;
    const long n = (long)s->np * s->dim;
    for (long iw = 0; iw < nw; ++iw) {
        double* w = walkers + iw * s->W;
        memset(w, 0, sizeof(double) * s->W);
        memcpy(POS(s, w), pos_aos + iw * n, sizeof(double) * n);
        build_tables(s, w);
        psi_evaluate(s, w);
        SC(s, w)[S_EL] = local_energy(s, w);
        SC(s, w)[S_ELI] = local_energy_imag(s, w);
        SC(s, w)[S_WEIGHT] = 1.0;
        SC(s, w)[S_ID] = 0.0;   /* Walker ids start at 0 (walker.h) */
    }
    return 0;
}

void o_refresh_all(const sys_t* s, double* w) {
    for (int d = 0; d < s->nbf; ++d) bf_refresh_all(s, w, d);
    if (s->cplx) return;   /* the complex determinant keeps its derivatives current */
    for (int b = 0; b < s->nblocks; ++b)
        for (int q = s->blocks[b].first; q < s->blocks[b].last; ++q) slater_refresh(s, w, q);
}

/* Refresh derivatives and recompute E_L of one walker (VMC/DMC measurement). */
void o_measure(void* p, double* w) {
    const sys_t* s = p;
    o_refresh_all(s, w);
    SC(s, w)[S_EL] = local_energy(s, w);
    SC(s, w)[S_ELI] = local_energy_imag(s, w);
}

/* ───────────────────────── one move ─────────────────────────────────── */

/* ratio of particle p at mv->new_pos: TrialWavefunction::ratio_batch. */
static void ratio(const sys_t* s, const double* w, int p, move_t* mv) {
    const int dim = s->dim, np = s->np;
    const double* pos = POS(s, w);
    /* pending distance row (update_batch) */
    for (int k = 0; k < np; ++k) {
        if (k == p) { mv->pend[k] = 0.0; continue; }
        double del[3];
        if (s->periodic) {
            mv->pend[k] = fold_dist(s, mv->new_pos, pos + k * dim, del);
        } else {
            double r2 = 0.0;
            for (int d = 0; d < dim; ++d) {
                const double diff = mv->new_pos[d] - pos[k * dim + d];
                r2 += diff * diff;
            }
            mv->pend[k] = sqrt(r2);
        }
    }
    for (int d = 0; d < dim; ++d) mv->new_grad[d] = mv->new_lap[d] = 0.0;
    for (int d = 0; d < dim; ++d) mv->new_pgrad[d] = mv->new_plap[d] = 0.0;
    mv->log_ratio = 0.0;
    mv->phase = 0.0;
    /* Slater */
    const int b = block_of(s, p);
    if (b >= 0 && s->cplx) {   /* ComplexSlaterDeterminant::ratio_batch */
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first, jrow = p - B->first;
        const double* Ar = w + s->o_A[b];
        const double* Ai = Ar + N * N;
        zc R = 0.0;
        for (int m = 0; m < N; ++m)
            R += CMPLX(Ar[m * N + jrow], Ai[m * N + jrow]) * corb(B, m, dim, mv->new_pos);
        const double absR = cabs(R);
        mv->log_ratio += log(fmax(absR, 1e-300));
        mv->phase += carg(R);
        const zc invR = absR > 0.0 ? 1.0 / R : 0.0;
        zc G[3], L[3];
        cderivs(s, w, b, jrow, mv->new_pos, G, L);
        for (int d = 0; d < dim; ++d) {
            /* cderivs gave L = Lraw - G²; the ratio wants Lraw/R - (G/R)² */
            const zc Lraw = L[d] + G[d] * G[d];
            const zc Gp = invR * G[d];
            const zc Lp = invR * Lraw - Gp * Gp;
            mv->new_grad[d] += creal(Gp);
            mv->new_lap[d] += creal(Lp);
            mv->new_pgrad[d] += cimag(Gp);
            mv->new_plap[d] += cimag(Lp);
        }
    } else if (b >= 0) {
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first, jrow = p - B->first;
        const double* A = w + s->o_A[b];
        orbitals(s, B, mv->new_pos, mv->nval, mv->ngrad, mv->nlap);
        double R = 0.0;
        for (int m = 0; m < N; ++m) R += A[m * N + jrow] * mv->nval[m];
        mv->log_ratio += log(fmax(fabs(R), 1e-300));
        if (R < 0.0) mv->phase += 3.14159265358979323846;
        const double invR = (R != 0.0) ? 1.0 / R : 0.0;
        for (int d = 0; d < dim; ++d) {
            double G = 0.0, Lraw = 0.0;
            for (int m = 0; m < N; ++m) {
                const double a = A[m * N + jrow];
                G += a * mv->ngrad[m * dim + d];
                Lraw += a * mv->nlap[m * dim + d];
            }
            const double Gp = invR * G;
            mv->new_grad[d] += Gp;
            mv->new_lap[d] += invR * Lraw - Gp * Gp;
        }
    }
    /* pair terms */
    int partners[1024];
    for (int t = 0; t < s->nterms; ++t) {
        const term_t* T = &s->terms[t];
        for (int d = 0; d < dim; ++d) mv->pg[t][d] = mv->pl[t][d] = 0.0;
        const int n = term_partners(T, p, partners);
        for (int q = 0; q < n; ++q) {
            const int k = partners[q];
            double del[3];
            for (int d = 0; d < dim; ++d) del[d] = mv->new_pos[d] - pos[k * dim + d];
            min_image(s, del);
            double* rad = mv->rad[t][k];
            radial(T, DIST(s, w)[p * np + k], &rad[0], &rad[1], &rad[2]);
            radial(T, mv->pend[k], &rad[3], &rad[4], &rad[5]);
            const double invr = 1.0 / mv->pend[k];
            mv->log_ratio += rad[3] - rad[0];
            for (int d = 0; d < dim; ++d) {
                const double dor = del[d] * invr;
                mv->pg[t][d] += rad[4] * dor;
                mv->pl[t][d] += rad[5] * dor * dor + rad[4] * invr * (1.0 - dor * dor);
            }
        }
        if (T->image) {
            const int same = t_same(T);
            const int in_a = p >= T->pairs[0][0] && p < T->pairs[0][1];
            const int in_b = !same && p >= T->pairs[0][2] && p < T->pairs[0][3];
            if (in_a || in_b) {
                const int nk = T->nk;
                const double* rho = w + s->o_rho[t];
                const double* pcache = w + s->o_pc[t];
                double* cn = mv->pc[t];
                double* sn = mv->ps[t];
                phases(s, T, mv->new_pos[0], mv->new_pos[1], cn, sn);
                const double* co = pcache + 2L * nk * t_slot(T, p);
                const double* so = co + nk;
                const double* mr = rho + (in_a ? 0 : 2 * nk);
                const double* mi = mr + nk;
                double dlog = 0.0;
                kterms_t kt;
                if (same) {
                    double qr[512], qi[512];
                    for (int k = 0; k < nk; ++k) {
                        qr[k] = mr[k] + cn[k] - co[k];
                        qi[k] = mi[k] + sn[k] - so[k];
                        dlog += T->w[k] * (qr[k] * qr[k] + qi[k] * qi[k] - mr[k] * mr[k] - mi[k] * mi[k]);
                    }
                    kt = kterms(T, cn, sn, qr, qi, 1.0);
                } else {
                    const double* orr = rho + (in_a ? 2 * nk : 0);
                    const double* oi = orr + nk;
                    for (int k = 0; k < nk; ++k)
                        dlog += 2.0 * T->w[k] * ((cn[k] - co[k]) * orr[k] + (sn[k] - so[k]) * oi[k]);
                    kt = kterms(T, cn, sn, orr, oi, 0.0);
                }
                mv->log_ratio += dlog;
                mv->pg[t][0] += kt.gx; mv->pg[t][1] += kt.gy;
                mv->pl[t][0] += kt.lx; mv->pl[t][1] += kt.ly;
            }
        }
        for (int d = 0; d < dim; ++d) {
            mv->new_grad[d] += mv->pg[t][d];
            mv->new_lap[d] += mv->pl[t][d];
        }
    }
    /* backflow determinants: BackflowSlaterDeterminant::ratio_batch, without the
       proposal Laplacian (the VMC/DMC drivers switch it off) */
    for (int d = 0; d < s->nbf; ++d) {
        const bfdet_t* D = &s->bf[d];
        mv->bused[d] = bf_affects(D, p);
        mv->bvalid[d] = 0;
        if (!mv->bused[d]) continue;
        const int N = D->last - D->first;
        static double pos2[2048];
        memcpy(pos2, pos, sizeof(double) * np * dim);
        const double old_r[2] = {pos[p * 2], pos[p * 2 + 1]};
        pos2[p * 2] = mv->new_pos[0];
        pos2[p * 2 + 1] = mv->new_pos[1];
        double* x = mv->bx[d];
        memcpy(x, w + D->o_x, sizeof(double) * N * 2);
        bf_shift(s, D, pos2, p, old_r, x);
        bf_particle_tables(s, D, pos2, p, x);
        bf_rows(s, D, x, g_bval, g_bgrad, g_bhess);
        memcpy(g_bwork, g_bval, sizeof(double) * N * N);
        const double* ls = w + D->o_ls;
        if (!bf_invert(N, g_bwork, mv->bA[d], &mv->bls[d][0], &mv->bls[d][1])) {
            mv->log_ratio += -700.0;
            mv->bg[d][0] = mv->bg[d][1] = 0.0;
            continue;
        }
        mv->bvalid[d] = 1;
        mv->log_ratio += mv->bls[d][0] - ls[0];
        if (mv->bls[d][1] * ls[1] < 0.0) mv->phase += 3.14159265358979323846;
        bf_f(N, mv->bA[d], g_bgrad, mv->bF[d]);
        bf_gradient(s, D, mv->bF[d], p, mv->bg[d]);
        mv->new_grad[0] += mv->bg[d][0];
        mv->new_grad[1] += mv->bg[d][1];
    }
}

/* Commit an accepted move of p: apply_move_batch_deferred of every component,
 * then WalkerSet::apply_move. */
static void commit(const sys_t* s, double* w, int p, move_t* mv) {
    const int dim = s->dim, np = s->np;
    double* pos = POS(s, w);
    double* bg = GRAD(s, w);
    double* bl = LAP(s, w);
    /* Slater, walker-tile path of apply_move_impl (deferred) */
    const int b = block_of(s, p);
    if (b >= 0 && s->cplx) {   /* ComplexSlaterDeterminant::apply_move_batch (eager) */
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first, jrow = p - B->first;
        double* Ar = w + s->o_A[b];
        double* Ai = Ar + N * N;
        double* bs = w + s->o_bs[b];
        zc D[64 * 64];
        crows(s, w, b, p, mv->new_pos, D);
        zc R = 0.0;
        for (int m = 0; m < N; ++m) R += CMPLX(Ar[m * N + jrow], Ai[m * N + jrow]) * D[jrow * N + m];
        const double dlog = log(fmax(cabs(R), 1e-300));
        bs[0] += dlog;
        LPC(s, w)[0] += dlog;
        SC(s, w)[S_LOGPSI] += dlog;
        int err = 0;
        cgj(N, D, Ar, Ai, &err);
        if (err) SC(s, w)[S_ERR] = 1.0;
        double* gc = GC(s, w, 0);
        double* lc = LC(s, w, 0);
        double* pgc = w + s->o_pgc;
        double* plc = w + s->o_plc;
        double* pgt = w + s->o_pgrad;
        double* plt = w + s->o_plap;
        for (int kr = 0; kr < N; ++kr) {
            const int part = B->first + kr;
            const double* r = part == p ? mv->new_pos : pos + part * dim;
            zc G[3], L[3];
            cderivs(s, w, b, kr, r, G, L);
            for (int d = 0; d < dim; ++d) {
                const int idx = part * dim + d;
                if (kr != jrow) {
                    bg[idx] += creal(G[d]) - gc[idx];
                    bl[idx] += creal(L[d]) - lc[idx];
                    pgt[idx] += cimag(G[d]) - pgc[idx];
                    plt[idx] += cimag(L[d]) - plc[idx];
                }
                gc[idx] = creal(G[d]);
                lc[idx] = creal(L[d]);
                pgc[idx] = cimag(G[d]);
                plc[idx] = cimag(L[d]);
            }
        }
    } else if (b >= 0) {
        const block_t* B = &s->blocks[b];
        const int N = B->last - B->first, jrow = p - B->first;
        double* A = w + s->o_A[b];
        double* D = w + s->o_D[b];
        double* Dg = w + s->o_Dg[b];
        double* Dl = w + s->o_Dl[b];
        double* rabs = w + s->o_rabs[b];
        double* bs = w + s->o_bs[b];
        double column[64], rowp[64];
        double ratio_ = 0.0, scale = 0.0;
        for (int m = 0; m < N; ++m) {
            const double term = A[m * N + jrow] * mv->nval[m];
            ratio_ += term;
            scale += fabs(term);
            column[m] = A[m * N + jrow];
        }
        for (int c = 0; c < N; ++c) {
            double prod = 0.0;
            for (int m = 0; m < N; ++m) prod += mv->nval[m] * A[m * N + c];
            rowp[c] = prod - (c == jrow ? 1.0 : 0.0);
        }
        for (int m = 0; m < N; ++m) {
            D[jrow * N + m] = mv->nval[m];
            for (int d = 0; d < dim; ++d) {
                Dg[(jrow * N + m) * dim + d] = mv->ngrad[m * dim + d];
                Dl[(jrow * N + m) * dim + d] = mv->nlap[m * dim + d];
            }
        }
        const double old_log = bs[0];
        bs[1] += 1.0;
        const int rebuild = bs[1] >= 64.0 || !isfinite(ratio_) || fabs(ratio_) < 1e-5 ||
                            bs[2] > 1e8 || fabs(ratio_) <= 1e4 * 2.220446049250313e-16 * scale;
        int err = 0;
        if (rebuild) {
            bs[0] = gj_rebuild(N, D, A, &err);
            bs[1] = 0.0;
        } else {
            bs[0] += log(fabs(ratio_));
            for (int a = 0; a < N; ++a) {
                const double factor = column[a] / ratio_;
                for (int c = 0; c < N; ++c) A[a * N + c] = A[a * N + c] - factor * rowp[c];
            }
        }
        double nd = 0.0, na = 0.0;
        for (int a = 0; a < N; ++a) {
            double rd_ = 0.0, ra = 0.0;
            for (int c = 0; c < N; ++c) {
                rd_ += fabs(D[a * N + c]);
                ra += fabs(A[a * N + c]);
            }
            if (rd_ > nd) nd = rd_;
            if (ra > na) na = ra;
            rabs[a] = rd_;
        }
        bs[2] = nd * na;
        if (!rebuild && (!isfinite(bs[2]) || bs[2] > 1e8)) {
            bs[0] = gj_rebuild(N, D, A, &err);
            bs[1] = 0.0;
        }
        if (err) SC(s, w)[S_ERR] = 1.0;
        const double dlog = bs[0] - old_log;
        LPC(s, w)[0] += dlog;
        SC(s, w)[S_LOGPSI] += dlog;
        /* the moved particle's own component cache (deferred partners) */
        double* gc = GC(s, w, 0);
        double* lc = LC(s, w, 0);
        for (int d = 0; d < dim; ++d) {
            double grad = 0.0, lap = 0.0;
            for (int m = 0; m < N; ++m) {
                const double a = A[m * N + jrow];
                grad += a * Dg[(jrow * N + m) * dim + d];
                lap += a * Dl[(jrow * N + m) * dim + d];
            }
            gc[p * dim + d] = grad;
            lc[p * dim + d] = lap - grad * grad;
        }
    }
    /* pair terms (eager) */
    int partners[1024];
    for (int t = 0; t < s->nterms; ++t) {
        const term_t* T = &s->terms[t];
        const int c = term_comp(s, t);
        double* gc = GC(s, w, c);
        double* lc = LC(s, w, c);
        const int n = term_partners(T, p, partners);
        int member = 0;
        for (int q = 0; q < T->npairs; ++q)
            if ((p >= T->pairs[q][0] && p < T->pairs[q][1]) || (p >= T->pairs[q][2] && p < T->pairs[q][3]))
                member = 1;
        if (!member) continue;
        for (int q = 0; q < n; ++q) {
            const int k = partners[q];
            double dold[3], dnew[3];
            for (int d = 0; d < dim; ++d) {
                dold[d] = pos[k * dim + d] - pos[p * dim + d];
                dnew[d] = pos[k * dim + d] - mv->new_pos[d];
            }
            min_image(s, dold);
            min_image(s, dnew);
            const double* rad = mv->rad[t][k];
            const double iro = 1.0 / DIST(s, w)[p * np + k];
            const double irn = 1.0 / mv->pend[k];
            const double dlog = rad[3] - rad[0];
            LPC(s, w)[c] += dlog;
            SC(s, w)[S_LOGPSI] += dlog;
            for (int d = 0; d < dim; ++d) {
                const double dor_old = dold[d] * iro, dor_new = dnew[d] * irn;
                const double g_old = rad[1] * dor_old, g_new = rad[4] * dor_new;
                const double dg = g_new - g_old;
                gc[k * dim + d] += dg;
                bg[k * dim + d] += dg;
                const double lap_old = rad[2] * dor_old * dor_old + rad[1] * iro * (1.0 - dor_old * dor_old);
                const double lap_new = rad[5] * dor_new * dor_new + rad[4] * irn * (1.0 - dor_new * dor_new);
                const double dl = lap_new - lap_old;
                lc[k * dim + d] += dl;
                bl[k * dim + d] += dl;
            }
        }
        if (T->image) {
            const int same = t_same(T);
            const int af = T->pairs[0][0], al = T->pairs[0][1], bf = T->pairs[0][2], bl_ = T->pairs[0][3];
            const int in_a = p >= af && p < al;
            const int in_b = !same && p >= bf && p < bl_;
            if (in_a || in_b) {
                const int nk = T->nk;
                double* rho = w + s->o_rho[t];
                double* pcache = w + s->o_pc[t];
                const double* cn = mv->pc[t];
                const double* sn = mv->ps[t];
                double* co = pcache + 2L * nk * t_slot(T, p);
                double* so = co + nk;
                double* mr = rho + (in_a ? 0 : 2 * nk);
                double* mi = mr + nk;
                double dr[512], di[512], dlog = 0.0;
                if (same) {
                    for (int k = 0; k < nk; ++k) {
                        dr[k] = cn[k] - co[k];
                        di[k] = sn[k] - so[k];
                        dlog += T->w[k] * (2.0 * (mr[k] * dr[k] + mi[k] * di[k]) + dr[k] * dr[k] + di[k] * di[k]);
                    }
                } else {
                    const double* orr = rho + (in_a ? 2 * nk : 0);
                    const double* oi = orr + nk;
                    for (int k = 0; k < nk; ++k) {
                        dr[k] = cn[k] - co[k];
                        di[k] = sn[k] - so[k];
                        dlog += 2.0 * T->w[k] * (dr[k] * orr[k] + di[k] * oi[k]);
                    }
                }
                LPC(s, w)[c] += dlog;
                SC(s, w)[S_LOGPSI] += dlog;
                const int sf = same ? af : (in_a ? bf : af), sl = same ? al : (in_a ? bl_ : al);
                for (int i = sf; i < sl; ++i) {
                    if (i == p) continue;
                    const double* ci = pcache + 2L * nk * t_slot(T, i);
                    kterms_t kt = kterms(T, ci, ci + nk, dr, di, 0.0);
                    gc[i * dim] += kt.gx; gc[i * dim + 1] += kt.gy;
                    bg[i * dim] += kt.gx; bg[i * dim + 1] += kt.gy;
                    lc[i * dim] += kt.lx; lc[i * dim + 1] += kt.ly;
                    bl[i * dim] += kt.lx; bl[i * dim + 1] += kt.ly;
                }
                for (int k = 0; k < nk; ++k) {
                    mr[k] += dr[k];
                    mi[k] += di[k];
                    co[k] = cn[k];
                    so[k] = sn[k];
                }
            }
        }
        /* p itself: absolute new values through the delta (pade_jastrow.cpp:610-633) */
        for (int d = 0; d < dim; ++d) {
            const double dgp = mv->pg[t][d] - gc[p * dim + d];
            const double dlp = mv->pl[t][d] - lc[p * dim + d];
            gc[p * dim + d] += dgp;
            bg[p * dim + d] += dgp;
            lc[p * dim + d] += dlp;
            bl[p * dim + d] += dlp;
        }
    }
    /* backflow determinants: the pending state becomes committed */
    for (int d = 0; d < s->nbf; ++d) {
        if (!mv->bused[d]) continue;
        const bfdet_t* D = &s->bf[d];
        const int N = D->last - D->first, c = bf_comp(s, d);
        if (!mv->bvalid[d]) SC(s, w)[S_ERR] = 1.0;
        memcpy(w + D->o_x, mv->bx[d], sizeof(double) * N * 2);
        memcpy(w + D->o_A, mv->bA[d], sizeof(double) * N * N);
        memcpy(w + D->o_F, mv->bF[d], sizeof(double) * N * 2);
        const double old = w[D->o_ls];
        w[D->o_ls] = mv->bls[d][0];
        w[D->o_ls + 1] = mv->bls[d][1];
        LPC(s, w)[c] = mv->bls[d][0];
        SC(s, w)[S_LOGPSI] += mv->bls[d][0] - old;
        for (int k = 0; k < 2; ++k) {
            GC(s, w, c)[p * 2 + k] = mv->bg[d][k];
            LC(s, w, c)[p * 2 + k] = 0.0;
        }
    }
    /* WalkerSet::apply_move: distance rows (masked commit form), position, wrap, grad/lap of p */
    double* dist = DIST(s, w);
    for (int k = 0; k < np; ++k) {
        if (k == p) continue;
        dist[p * np + k] += 1.0 * (mv->pend[k] - dist[p * np + k]);
        dist[k * np + p] += 1.0 * (mv->pend[k] - dist[k * np + p]);
    }
    for (int d = 0; d < dim; ++d) pos[p * dim + d] = mv->new_pos[d];
    wrap(s, pos + p * dim);
    for (int d = 0; d < dim; ++d) {
        bg[p * dim + d] = mv->new_grad[d];
        bl[p * dim + d] = mv->new_lap[d];
    }
    if (s->cplx)
        for (int d = 0; d < dim; ++d) {
            w[s->o_pgrad + p * dim + d] = mv->new_pgrad[d];
            w[s->o_plap + p * dim + d] = mv->new_plap[d];
        }
}

/*
 * Single move for the component-level parity tests: propose p at new_pos,
 * report (log_ratio, phase, new_grad[dim], new_lap[dim]) in out, and commit
 * when accept != 0.
 */
static move_t g_mv;
int o_move(void* ps, double* w, int p, const double* new_pos, int accept, double* out) {
    const sys_t* s = ps;
    move_t* mv = &g_mv;
    for (int d = 0; d < s->dim; ++d) mv->new_pos[d] = new_pos[d];
    ratio(s, w, p, mv);
    out[0] = mv->log_ratio;
    out[1] = mv->phase;
    for (int d = 0; d < s->dim; ++d) {
        out[2 + d] = mv->new_grad[d];
        out[2 + s->dim + d] = mv->new_lap[d];
    }
    if (accept) commit(s, w, p, mv);
    return 0;
}

/* ───────────────────────── drivers ──────────────────────────────────── */

/* One crowd's sweep randoms, sweep_blocking.h:39-48 order. */
static void draw_randoms(xo_t* rng, int np, int dim, long n, double* buf) {
    for (int p = 0; p < np; ++p) {
        double* row = buf + (long)p * (dim + 1) * n;
        for (int d = 0; d < dim; ++d)
            for (long w = 0; w < n; ++w) row[d * n + w] = xo_gaussian(rng);
        for (long w = 0; w < n; ++w) row[dim * n + w] = xo_uniform(rng);
    }
}

static double umrigar(double tm, double vsq) {
    if (vsq < 1e-10) return tm;
    return (-1.0 + sqrt(1.0 + 2.0 * 1.0 * tm * vsq)) / (1.0 * vsq);
}

/* VMC sweep of one walker (vmc.cpp:82-155), reading its column of the crowd's
 * randoms (n walkers in the crowd, this walker at index iw). */
static long vmc_sweep_walker(const sys_t* s, double* w, const double* rnd, long n, long iw,
                             double tau, int drift) {
    const int np = s->np, dim = s->dim;
    long acc = 0;
    move_t* mv = &g_mv;
    for (int p = 0; p < np; ++p) {
        if (drift) {
            slater_refresh(s, w, p);
            for (int d = 0; d < s->nbf; ++d) bf_refresh_particle(s, w, d, p);
        }
        const double* gauss = rnd + (long)p * (dim + 1) * n;
        const double u = gauss[dim * n + iw];
        for (int d = 0; d < dim; ++d) {
            const double tm = tau * s->inv_mass[p * dim + d];
            const double sig = sqrt(tm);
            mv->new_pos[d] = drift ? POS(s, w)[p * dim + d] + tm * GRAD(s, w)[p * dim + d] +
                                         sig * gauss[d * n + iw]
                                   : POS(s, w)[p * dim + d] + sig * gauss[d * n + iw];
        }
        ratio(s, w, p, mv);
        int accept;
        if (drift) {
            double log_corr = 0.0;
            for (int d = 0; d < dim; ++d) {
                const double tm = tau * s->inv_mass[p * dim + d];
                const double delta = mv->new_pos[d] - POS(s, w)[p * dim + d];
                const double go = GRAD(s, w)[p * dim + d], gn = mv->new_grad[d];
                log_corr += -delta * (go + gn) + 0.5 * tm * (go * go - gn * gn);
            }
            const double la = 2.0 * mv->log_ratio + log_corr;
            accept = la >= 0.0 || u < exp(la);
        } else {
            accept = u < exp(2.0 * mv->log_ratio);
        }
        if (accept) {
            ++acc;
            commit(s, w, p, mv);
        }
    }
    return acc;
}

/*
 * VMC::run restated: nt = min(threads, nw) streams stream_seed(seed,
 * "vmc-thrd", t) over contiguous even splits; per step n_substeps sweeps,
 * refresh, E_L.  el_out[(step_global) * nw + w] for every step, equilibration
 * included (eq steps first).  stats: [accepted, proposed].
 */
int o_vmc(void* ps, double* walkers, long nw, int threads, uint64_t seed, int n_eq, int n_acc,
          int n_steps, int n_substeps, double tau, int drift, double* el_out, double* stats) {
    const sys_t* s = ps;
    const int nt = threads < nw ? threads : (int)nw;
    const long base = nw / nt, rem = nw % nt;
    const int np = s->np, dim = s->dim;
    double* rnd = malloc(sizeof(double) * (size_t)np * (dim + 1) * (base + 1));
    long accepted = 0, proposed = 0;
    long w0 = 0;
    for (int t = 0; t < nt; ++t) {
        const long n = base + (t < rem ? 1 : 0);
        xo_t rng;
        xo_seed(&rng, o_stream_seed(seed, 0x766d632d74687264ULL, (uint64_t)t));
        long step = 0;
        for (int blk = 0; blk < n_eq + n_acc; ++blk)
            for (int st = 0; st < n_steps; ++st, ++step) {
                for (int sub = 0; sub < n_substeps; ++sub) {
                    draw_randoms(&rng, np, dim, n, rnd);
                    long a = 0;
                    for (long iw = 0; iw < n; ++iw)
                        a += vmc_sweep_walker(s, walkers + (w0 + iw) * s->W, rnd, n, iw, tau, drift);
                    if (blk >= n_eq) {   /* vmc.cpp counts the accumulation only */
                        accepted += a;
                        proposed += n * np;
                    }
                }
                for (long iw = 0; iw < n; ++iw) {
                    double* w = walkers + (w0 + iw) * s->W;
                    o_measure(ps, w);
                    if (el_out) el_out[step * nw + w0 + iw] = SC(s, w)[S_EL];
                }
            }
        w0 += n;
    }
    free(rnd);
    stats[0] = (double)accepted;
    stats[1] = (double)proposed;
    return 0;
}

/* DMC sweep of one walker (dmc.cpp:203-337), bare reweighting. */
static long dmc_sweep_walker(const sys_t* s, double* w, const double* rnd, long stride, long iw,
                             double tau) {
    const int np = s->np, dim = s->dim;
    long acc = 0;
    move_t* mv = &g_mv;
    double* sc = SC(s, w);
    for (int p = 0; p < np; ++p) {
        slater_refresh(s, w, p);
        for (int d = 0; d < s->nbf; ++d) bf_refresh_particle(s, w, d, p);
        const double tm_p = tau * s->inv_mass[p * dim];
        const double* gauss = rnd + (long)p * (dim + 1) * stride;
        const double u = gauss[dim * stride + iw];
        double vsq = 0.0;
        for (int d = 0; d < dim; ++d) vsq += GRAD(s, w)[p * dim + d] * GRAD(s, w)[p * dim + d];
        const double sc_fwd = umrigar(tm_p, vsq);
        for (int d = 0; d < dim; ++d) {
            const double sig = sqrt(tau * s->inv_mass[p * dim + d]);
            mv->new_pos[d] = POS(s, w)[p * dim + d] + sc_fwd * GRAD(s, w)[p * dim + d] + sig * gauss[d * stride + iw];
        }
        ratio(s, w, p, mv);
        int accept = 0;
        /* fixed node: a sign change rejects; fixed phase (complex ψ): no gate */
        if (s->cplx || !(cos(mv->phase) < 2.220446049250313e-16)) {
            double vn = 0.0;
            for (int d = 0; d < dim; ++d) vn += mv->new_grad[d] * mv->new_grad[d];
            const double sc_bwd = umrigar(tm_p, vn);
            double log_corr = 0.0;
            for (int d = 0; d < dim; ++d) {
                const double tm = tau * s->inv_mass[p * dim + d];
                const double delta = mv->new_pos[d] - POS(s, w)[p * dim + d];
                const double df = sc_fwd * GRAD(s, w)[p * dim + d];
                const double db = sc_bwd * mv->new_grad[d];
                log_corr += tm <= 0.0 ? 0.0 : (-delta * (df + db) + 0.5 * (df * df - db * db)) / tm;
            }
            const double la = 2.0 * mv->log_ratio + log_corr;
            const double pacc = la >= 0.0 ? 1.0 : exp(la);
            accept = la >= 0.0 || u < pacc;
        }
        double rr = 0.0;
        for (int d = 0; d < dim; ++d) {
            const double tm = tau * s->inv_mass[p * dim + d];
            const double dr = mv->new_pos[d] - POS(s, w)[p * dim + d];
            rr += tm * dr * dr;
        }
        sc[S_RRP] += rr;
        if (accept) {
            sc[S_RRA] += rr;
            ++acc;
            commit(s, w, p, mv);
        }
    }
    return acc;
}

static int cmp_dbl(const void* a, const void* b) {
    const double x = *(const double*)a, y = *(const double*)b;
    return x < y ? -1 : x > y;
}
/* median of n values as nth_element-based median_in_place (statistics.cpp) */
static double median(double* v, long n) {
    qsort(v, (size_t)n, sizeof(double), cmp_dbl);
    if (n % 2) return v[n / 2];
    return 0.5 * (v[n / 2 - 1] + v[n / 2]);
}

/*
 * DMC::run restated (bare reweighting, universal cutoff, alpha = 2): per step
 * every crowd advances its walkers, then the population branches on the
 * serial branch stream.  walkers must hold capacity records.  trace gets per
 * step [nw_before_branch, sum w E, sum w, e_trial_after, n_accepted].
 */
int o_dmc(void* ps, double* walkers, long* nw_io, long capacity, int threads, uint64_t seed,
          int n_eq, int n_acc, int n_steps, int n_substeps, double tau, double generations,
          long target, double* trace, double* el_trace, long el_trace_cap) {
    const sys_t* s = ps;
    const int np = s->np, dim = s->dim;
    long nw = *nw_io;
    const long W = s->W;
    const int nthreads = threads < nw ? threads : (int)nw;
    xo_t* rngs = malloc(sizeof(xo_t) * nthreads);
    for (int t = 0; t < nthreads; ++t)
        xo_seed(&rngs[t], o_stream_seed(seed, 0x646d632d74687264ULL, (uint64_t)t));
    xo_t brng;
    xo_seed(&brng, o_stream_seed(seed, 0x646d632d62726368ULL, 0));
    const long cap = (2 * target + 2) > nw ? (2 * target + 2) : nw;
    if (capacity < cap) { free(rngs); return -1; }
    double* rnd = malloc(sizeof(double) * (size_t)np * (dim + 1) * cap);
    double* scratch = malloc(sizeof(double) * (size_t)cap);
    double* tmpw = malloc(sizeof(double) * (size_t)W * cap);
    long* src = malloc(sizeof(long) * (size_t)(2 * target + 2 + cap));
    /* diffusing particles: inv_mass >= 1e-3 max (dmc.cpp:50-66) */
    double max_inv = 0.0;
    for (int i = 0; i < np * dim; ++i) if (s->inv_mass[i] > max_inv) max_inv = s->inv_mass[i];
    long n_diff = 0;
    for (int g = 0; g < s->ngroups; ++g) {
        double gi = 0.0;
        for (int d = 0; d < dim; ++d) if (s->inv_mass[s->gfirst[g] * dim + d] > gi) gi = s->inv_mass[s->gfirst[g] * dim + d];
        if (gi >= 1e-3 * max_inv) n_diff += s->glast[g] - s->gfirst[g];
    }
    if (n_diff < 1) n_diff = 1;
    /* population control */
    const double t_step = tau * (n_substeps > 1 ? n_substeps : 1);
    const double feedback = (t_step > 0.0 && generations > 0.0) ? 1.0 / (generations * t_step) : 0.0;
    double e_sum0 = 0.0;
    for (long i = 0; i < nw; ++i) e_sum0 += SC(s, walkers + i * W)[S_EL];
    double etrial = e_sum0 / (double)nw, eref = etrial, eref_sum = 0.0, eref_wsum = 0.0;
    double e_cut = INFINITY, e_max = INFINITY;
    const double alpha = 2.0;
    long next_id = 0;
    for (long i = 0; i < nw; ++i) {
        const double id = SC(s, walkers + i * W)[S_ID];
        if ((long)id + 1 > next_id) next_id = (long)id + 1;
    }
    /* energy spread of the starting population */
    #define SET_SPREAD() do { \
        for (long i_ = 0; i_ < nw; ++i_) scratch[i_] = SC(s, walkers + i_ * W)[S_EL]; \
        const double centre_ = median(scratch, nw); \
        for (long i_ = 0; i_ < nw; ++i_) scratch[i_] = fabs(SC(s, walkers + i_ * W)[S_EL] - centre_); \
        const double sigma_ = 1.4826 * median(scratch, nw); \
        if (!(isfinite(sigma_) && sigma_ > 0.0 && tau > 0.0)) { e_cut = INFINITY; e_max = INFINITY; } \
        else { e_cut = alpha * sqrt(sigma_ * sqrt((double)n_diff) / tau); e_max = 1.5 * e_cut; } \
    } while (0)
    SET_SPREAD();
    long step_index = 0, el_rows = 0;
    for (int blk = 0; blk < n_eq + n_acc; ++blk) {
        const int measure = blk >= n_eq;
        if (blk == n_eq) { eref_sum = 0.0; eref_wsum = 0.0; }
        for (int st = 0; st < n_steps; ++st, ++step_index) {
            const int nact = nthreads < nw ? nthreads : (int)nw;
            const long base = nw / nact, rem = nw % nact;
            double e = 0.0, wsum = 0.0;
            long acc = 0;
            for (int t = 0; t < nact; ++t) {
                const long w0 = t * base + (t < rem ? t : rem);
                const long cnt = base + (t < rem ? 1 : 0);
                for (long i = w0; i < w0 + cnt; ++i) {
                    double* sc = SC(s, walkers + i * W);
                    sc[S_RRP] = 0.0; sc[S_RRA] = 0.0; sc[S_WEIGHT] = 1.0; sc[S_EPREV] = sc[S_EL];
                }
                for (int sub = 0; sub < n_substeps; ++sub) {
                    /* draw_sweep_randoms with stride = capacity over [w0, w0+cnt) */
                    for (int p = 0; p < np; ++p) {
                        double* row = rnd + (long)p * (dim + 1) * cap;
                        for (int d = 0; d < dim; ++d)
                            for (long i = w0; i < w0 + cnt; ++i) row[d * cap + i] = xo_gaussian(&rngs[t]);
                        for (long i = w0; i < w0 + cnt; ++i) row[dim * cap + i] = xo_uniform(&rngs[t]);
                    }
                    for (long i = w0; i < w0 + cnt; ++i)
                        acc += dmc_sweep_walker(s, walkers + i * W, rnd, cap, i, tau);
                    for (long i = w0; i < w0 + cnt; ++i) {
                        double* w = walkers + i * W;
                        o_measure(ps, w);
                        double* sc = SC(s, w);
                        const double enew = sc[S_EL], eold = sc[S_EPREV];
                        double half_tau = 0.5 * tau;
                        const double x = fmax(eref - enew, eref - eold);
                        if (x > e_max) half_tau = 0.0;
                        else if (x > e_cut) half_tau *= 1.0 - (x - e_cut) / (e_max - e_cut);
                        sc[S_WEIGHT] *= exp(half_tau * (2.0 * etrial - enew - eold));
                        sc[S_EPREV] = enew;
                    }
                }
                for (long i = w0; i < w0 + cnt; ++i) {
                    double* sc = SC(s, walkers + i * W);
                    if (tau > 0.0) sc[S_AGE] = sc[S_RRP] > 0.0 ? 0.0 : sc[S_AGE] + 1.0;
                    e += sc[S_WEIGHT] * sc[S_EL];
                    wsum += sc[S_WEIGHT];
                }
            }
            if (el_trace && el_rows < el_trace_cap) {
                el_trace[el_rows * 2] = (double)nw;
                el_trace[el_rows * 2 + 1] = e;
                ++el_rows;
            }
            const double ens_e = wsum > 0.0 ? e / wsum : etrial;
            /* branch (walker_set.cpp:187-239) */
            long ns = 0;
            for (long i = 0; i < nw; ++i) {
                const int m = (int)(SC(s, walkers + i * W)[S_WEIGHT] + xo_uniform(&brng));
                for (int c = 0; c < m; ++c) src[ns++] = i;
            }
            const long n_max = 2 * target + 1, n_min = target / 5 + 1;
            if (ns == 0) {
                long best = 0;
                for (long i = 1; i < nw; ++i)
                    if (SC(s, walkers + i * W)[S_WEIGHT] > SC(s, walkers + best * W)[S_WEIGHT]) best = i;
                src[ns++] = best;
            }
            while (ns > n_max) {
                const long i = (long)(xo_uniform(&brng) * (double)ns);
                src[i] = src[ns - 1];
                --ns;
            }
            while (ns < n_min) {
                const long i = (long)(xo_uniform(&brng) * (double)ns);
                src[ns++] = src[i];
            }
            char* seen = calloc((size_t)nw, 1);
            for (long j = 0; j < ns; ++j) memcpy(tmpw + j * W, walkers + src[j] * W, sizeof(double) * W);
            for (long j = 0; j < ns; ++j) {
                double* sc = SC(s, tmpw + j * W);
                if (seen[src[j]]) {
                    sc[S_PARENT] = sc[S_ID];
                    sc[S_ID] = (double)next_id++;
                } else {
                    seen[src[j]] = 1;
                }
                sc[S_WEIGHT] = 1.0;
            }
            free(seen);
            memcpy(walkers, tmpw, sizeof(double) * W * ns);
            const long nw_before = nw;
            nw = ns;
            /* population update */
            if (measure) {
                eref_sum += ens_e * wsum;
                eref_wsum += wsum;
                if (eref_wsum > 0.0) eref = eref_sum / eref_wsum;
            } else {
                eref = ens_e;
            }
            if (wsum > 0.0) etrial = eref - feedback * log(wsum / (double)target);
            if (trace) {
                double* tr = trace + step_index * 5;
                tr[0] = (double)nw_before;
                tr[1] = e;
                tr[2] = wsum;
                tr[3] = etrial;
                tr[4] = (double)acc;
            }
        }
        if (!measure) SET_SPREAD();
    }
    #undef SET_SPREAD
    *nw_io = nw;
    free(rnd); free(scratch); free(tmpw); free(src); free(rngs);
    return 0;
}

/* ───────────────────────── estimators ───────────────────────────────────
 * One measurement of the observable estimators on nw configurations, SoA
 * positions [p*dim*nw + d*nw + w], configuration w weighted by wts[w]; the
 * histograms and accumulators are added to (the caller zeroes them at a
 * block start), *wsum receives += Σ_w wts[w] in walker order. */

/* Triangular index of an unordered group pair
 * (src/estimators/pair_correlation.cpp:88-93). */
static long est_pair_id(long ga, long gb, long ng) {
    if (gb < ga) { const long t = ga; ga = gb; gb = t; }
    return ga * ng - ga * (ga - 1) / 2 + (gb - ga);
}

static int est_group_of(const sys_t* s, int p) {
    for (int g = 0; g < s->ngroups; ++g)
        if (p >= s->gfirst[g] && p < s->glast[g]) return g;
    return 0;
}

/* PairCorrelation::accumulate (src/estimators/pair_correlation.cpp:99-127):
 * pairs i < j in order, walkers innermost; the distance is the one the
 * distance table holds after build_all (batched_distance_table.cpp:20-55):
 * minimum image of r_i - r_j, squares summed over dimensions in order. */
void o_est_gofr(void* ps, const double* pos, long nw, const double* wts, double rmax, int n_bins,
                double* hist, double* wsum) {
    const sys_t* s = (const sys_t*)ps;
    const int np = s->np, dim = s->dim;
    const double inv_delta = (double)n_bins / rmax;
    for (int i = 0; i < np; ++i) {
        const int gi = est_group_of(s, i);
        for (int j = i + 1; j < np; ++j) {
            double* h = hist + est_pair_id(gi, est_group_of(s, j), s->ngroups) * n_bins;
            for (long w = 0; w < nw; ++w) {
                double xi[3], xj[3], del[3];
                for (int d = 0; d < dim; ++d) {
                    xi[d] = pos[((long)i * dim + d) * nw + w];
                    xj[d] = pos[((long)j * dim + d) * nw + w];
                }
                const double r = fold_dist(s, xi, xj, del);
                if (r < rmax) {
                    const size_t bin = (size_t)(r * inv_delta);
                    if (bin < (size_t)n_bins) h[bin] += wts[w];
                }
            }
        }
    }
    double t = 0.0;
    for (long w = 0; w < nw; ++w) t += wts[w];
    *wsum += t;
}

/* Density::accumulate (src/estimators/density.cpp:70-130): per group (or per
 * particle when per_particle), a cell of the n_bins^dim grid per particle;
 * periodic cells bin the fractional coordinates of the wrapped position,
 * open ones the box [-rmax, rmax)^dim. */
void o_est_density(void* ps, const double* pos, long nw, const double* wts, double rmax, int n_bins,
                   int per_particle, double* hist, double* wsum) {
    const sys_t* s = (const sys_t*)ps;
    const int dim = s->dim;
    size_t n_cells = 1;
    for (int d = 0; d < dim; ++d) n_cells *= (size_t)n_bins;
    const double two_rmax = 2.0 * rmax;
    const double inv_delta = (double)n_bins / (2.0 * rmax);
    const int nser = per_particle ? s->np : s->ngroups;
    for (int g = 0; g < nser; ++g) {
        double* h = hist + (size_t)g * n_cells;
        const int first = per_particle ? g : s->gfirst[g];
        const int last = per_particle ? g + 1 : s->glast[g];
        for (int p = first; p < last; ++p) {
            const double* base = pos + (long)p * dim * nw;
            for (long w = 0; w < nw; ++w) {
                size_t cell = 0;
                if (s->periodic) {
                    double r[3] = {0, 0, 0}, f[3] = {0, 0, 0};
                    for (int d = 0; d < dim; ++d) r[d] = base[d * nw + w];
                    wrap(s, r);
                    for (int i = 0; i < dim; ++i) {
                        double acc = 0.0;
                        for (int d = 0; d < dim; ++d) acc += s->ainv[i * dim + d] * r[d];
                        f[i] = acc;
                    }
                    for (int d = 0; d < dim; ++d) {
                        const double x = f[d] + 0.5;
                        size_t b = (size_t)(x * (double)n_bins);
                        if (b >= (size_t)n_bins) b = (size_t)n_bins - 1;
                        cell = cell * (size_t)n_bins + b;
                    }
                    h[cell] += wts[w];
                    continue;
                }
                int in_box = 1;
                for (int d = 0; d < dim; ++d) {
                    const double x = base[d * nw + w] + rmax;
                    if (x < 0.0 || x >= two_rmax) {
                        in_box = 0;
                        break;
                    }
                    size_t b = (size_t)(x * inv_delta);
                    if (b >= (size_t)n_bins) b = (size_t)n_bins - 1;
                    cell = cell * (size_t)n_bins + b;
                }
                if (in_box) h[cell] += wts[w];
            }
        }
    }
    double t = 0.0;
    for (long w = 0; w < nw; ++w) t += wts[w];
    *wsum += t;
}

/* e^{inθ}, n = 0..m, by the recurrence of numerics::ReciprocalPhases::ladder
 * (src/numerics/reciprocal_phases.h:62-76). */
static void est_ladder(double theta, int m, double* re, double* im) {
    const double c = cos(theta), sn = sin(theta);
    re[0] = 1.0;
    im[0] = 0.0;
    for (int n = 1; n <= m; ++n) {
        re[n] = re[n - 1] * c - im[n - 1] * sn;
        im[n] = re[n - 1] * sn + im[n - 1] * c;
    }
}

/* StructureFactor::accumulate (src/estimators/structure_factor.cpp:80-121):
 * per walker the group densities ρ_g(k) = Σ_i e^{ik·r_i} (ReciprocalPhases,
 * reciprocal_phases.h:41-58), then acc_re/acc_im += w ρ_g, and for every
 * group pair a <= b acc_s += w (Re ρ_a Re ρ_b + Im ρ_a Im ρ_b). */
void o_est_sofk(void* ps, const double* pos, long nw, const double* wts, int nk, const int* n1,
                const int* n2, double* acc_s, double* acc_re, double* acc_im, double* wsum) {
    const sys_t* s = (const sys_t*)ps;
    const int ng = s->ngroups;
    int m1 = 0, m2 = 0;
    for (int k = 0; k < nk; ++k) {
        if (abs(n1[k]) > m1) m1 = abs(n1[k]);
        if (abs(n2[k]) > m2) m2 = abs(n2[k]);
    }
    const double b1x = s->recip[0], b1y = s->recip[1], b2x = s->recip[2], b2y = s->recip[3];
    double* e1r = malloc(sizeof(double) * (m1 + 1));
    double* e1i = malloc(sizeof(double) * (m1 + 1));
    double* e2r = malloc(sizeof(double) * (m2 + 1));
    double* e2i = malloc(sizeof(double) * (m2 + 1));
    double* rr = malloc(sizeof(double) * ng * nk);
    double* ri = malloc(sizeof(double) * ng * nk);
    for (long w = 0; w < nw; ++w) {
        const double wt = wts[w];
        for (int g = 0; g < ng; ++g) {
            double* re = rr + g * nk;
            double* im = ri + g * nk;
            for (int k = 0; k < nk; ++k) re[k] = im[k] = 0.0;
            for (int i = s->gfirst[g]; i < s->glast[g]; ++i) {
                const double x = pos[((long)i * 2 + 0) * nw + w], y = pos[((long)i * 2 + 1) * nw + w];
                est_ladder(b1x * x + b1y * y, m1, e1r, e1i);
                est_ladder(b2x * x + b2y * y, m2, e2r, e2i);
                for (int k = 0; k < nk; ++k) {
                    const int a = n1[k], b = n2[k];
                    const double ar = e1r[abs(a)], ai = a < 0 ? -e1i[-a] : e1i[a];
                    const double br = e2r[abs(b)], bi = b < 0 ? -e2i[-b] : e2i[b];
                    const double c = ar * br - ai * bi;
                    const double sn = ar * bi + ai * br;
                    re[k] += c;
                    im[k] += sn;
                }
            }
            for (int k = 0; k < nk; ++k) {
                acc_re[g * nk + k] += wt * re[k];
                acc_im[g * nk + k] += wt * im[k];
            }
        }
        int pid = 0;
        for (int a = 0; a < ng; ++a)
            for (int b = a; b < ng; ++b, ++pid) {
                const double *ra = rr + a * nk, *ia = ri + a * nk, *rb = rr + b * nk, *ib = ri + b * nk;
                for (int k = 0; k < nk; ++k) acc_s[pid * nk + k] += wt * (ra[k] * rb[k] + ia[k] * ib[k]);
            }
        *wsum += wt;
    }
    free(e1r); free(e1i); free(e2r); free(e2i); free(rr); free(ri);
}
