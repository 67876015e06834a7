// C ABI of the B200 walker hot path (include/alea_gpu.h): context and device
// buffers, the system description on the device, and the host halves of the
// VMC/DMC drivers (population control, branching, statistics).
//
// Host algorithms restated from the reference (ItaloAlb/alea):
//   streams        src/numerics/random.h:39-56, src/numerics/xoshiro_random.h:23-49
//   ziggurat       src/numerics/xoshiro_random.h:110-175 (table construction)
//   cell           src/population/simulation_cell.cpp:160-270
//   VMC loop       src/qmc/vmc.cpp:23-62, :189-431
//   DMC loop       src/qmc/dmc.cpp:525-884, src/qmc/population_control.cpp:37-103
//   branching      src/population/walker_set.cpp:187-239
//   spread         src/numerics/statistics.cpp:297-315
#include <algorithm>
#include <atomic>
#include <mutex>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <map>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/alea_gpu.h"
#include "alea_internal.h"
#include "alea_dev.cuh"
#include "alea_estimators.h"
#include "alea_kernels.h"

using namespace alea_gpu;

namespace {

thread_local std::string g_create_error;   // per host thread, as the ABI reads it

// ───────────────────────── host random numbers ─────────────────────────

uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ULL;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}
uint64_t stream_seed(uint64_t base, uint64_t stream, uint64_t index) {
    return splitmix64(splitmix64(splitmix64(base) ^ stream) ^ index);
}
struct HostXo {
    uint64_t s[4];
    explicit HostXo(uint64_t seed) {
        for (uint64_t i = 0; i < 4; ++i) s[i] = splitmix64(seed + i * 0x9e3779b97f4a7c15ULL);
    }
    HostXo() : s{0, 0, 0, 0} {}
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t result = rotl(s[0] + s[3], 23) + s[0];
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    double uniform() { return static_cast<double>(static_cast<int64_t>(next() >> 11)) * 0x1.0p-53; }
};

// Ziggurat tables of 256 equal-area regions under exp(-x²/2), 2⁵² fixed point
// (Marsaglia & Tsang 2000; region/sign/position split after Doornik 2005):
// the tail start r solves "the top layer closes at f = 1" by bisection.
struct Ziggurat {
    uint64_t k[256];
    double w[256], f[256], r;
};
Ziggurat make_ziggurat() {
    auto f = [](double x) { return std::exp(-0.5 * x * x); };
    auto v_of = [&](double r) {
        return r * f(r) + std::sqrt(0.5 * 3.14159265358979323846) * std::erfc(r / 1.41421356237309504880);
    };
    double x[256] = {};
    auto mismatch = [&](double r) {
        const double v = v_of(r);
        x[255] = r;
        for (int i = 255; i >= 2; --i) {
            const double y = f(x[i]) + v / x[i];
            if (y >= 1.0) return 1.0;
            x[i - 1] = std::sqrt(-2.0 * std::log(y));
        }
        return f(x[1]) + v / x[1] - 1.0;
    };
    double lo = 3.0, hi = 4.5;
    for (;;) {
        const double mid = 0.5 * (lo + hi);
        if (mid == lo || mid == hi) break;
        (mismatch(mid) > 0.0 ? lo : hi) = mid;
    }
    Ziggurat z{};
    z.r = hi;
    (void)mismatch(z.r);
    const double two52 = 0x1.0p52;
    const double base = v_of(z.r) / f(z.r);
    z.k[0] = static_cast<uint64_t>(two52 * (z.r / base));
    z.w[0] = base / two52;
    z.f[0] = 1.0;
    for (int i = 1; i < 256; ++i) {
        z.k[i] = i == 1 ? 0 : static_cast<uint64_t>(two52 * (x[i - 1] / x[i]));
        z.w[i] = x[i] / two52;
        z.f[i] = f(x[i]);
    }
    return z;
}

double median_in_place(std::vector<double>& v) {
    const std::size_t n = v.size(), mid = n / 2;
    std::nth_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(mid), v.end());
    const double upper = v[mid];
    if (n % 2 == 1) return upper;
    const double lower = *std::max_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(mid));
    return 0.5 * (lower + upper);
}
double robust_spread(const double* x, std::size_t n) {
    if (n == 0) return 0.0;
    std::vector<double> s(x, x + n);
    const double centre = median_in_place(s);
    for (std::size_t i = 0; i < n; ++i) s[i] = std::abs(x[i] - centre);
    return 1.4826 * median_in_place(s);
}

// Flyvbjerg-Petersen blocking: standard error at each pairwise level; the
// estimate is the largest one among levels that keep at least 8 blocks.
void reblock(const std::vector<double>& series, double& mean, double& err) {
    mean = 0.0;
    err = 0.0;
    if (series.empty()) return;
    for (double x : series) mean += x;
    mean /= static_cast<double>(series.size());
    std::vector<double> cur = series;
    while (cur.size() >= 8) {
        const double n = static_cast<double>(cur.size());
        double m = 0.0, v = 0.0;
        for (double x : cur) m += x;
        m /= n;
        for (double x : cur) v += (x - m) * (x - m);
        v /= (n - 1.0);
        err = std::max(err, std::sqrt(v / n));
        std::vector<double> next(cur.size() / 2);
        for (std::size_t i = 0; i < next.size(); ++i) next[i] = 0.5 * (cur[2 * i] + cur[2 * i + 1]);
        cur.swap(next);
    }
}

}  // namespace

// ───────────────────────── context ──────────────────────────────────────

// Forward walking (src/qmc/forward_walking.h): a ring of position snapshots
// in device memory, the ancestry of every live walker in each snapshot on the
// host (integers, carried through each branch's src map), per-lag pure
// estimators and potential-energy block sums.
struct FwSlot {
    long step = -1;                // the step it was taken at; -1: unused
    int nw = 0;
    double* d_pos = nullptr;       // [capacity][np * 2]
    std::vector<int> anc;          // [live walkers]: index into the snapshot
};

struct FwState {
    std::vector<double> lags;      // imaginary times, as set
    int interval = 1;
    std::vector<alea_gpu::EstimatorSet*> est;   // per lag
    // per run
    std::vector<long> lag_steps;
    double step_time = 0.0;
    long first_measured = 0, first_snapshot = 0;
    std::vector<FwSlot> slots;
    std::vector<double> blk_wpot, blk_w;
    std::vector<std::vector<double>> block_pot;
    std::vector<int64_t> measurements;
    std::vector<double> surviving;
    int* d_idx = nullptr;          // kept ancestors [capacity]
    double* d_kw = nullptr;        // their descendant weights
    double* d_v = nullptr;         // their potentials
};

struct alea_gpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    DevSys sys{};
    void* arena = nullptr;
    int capacity = 0, nw = 0;
    double* rec[2] = {nullptr, nullptr};
    int cur = 0;
    double* randoms = nullptr;
    int rnd_sweeps = 0;
    uint64_t* streams = nullptr;
    int n_streams = 0, streams_cap = 0;
    int2* pairs = nullptr;
    int npair = 0;
    double* d_buf = nullptr;       // staging [max(np*dim, 8) * capacity]
    double* d_sigma = nullptr;     // [np*dim]
    double sigma_tau = -1.0;
    int* d_src = nullptr;
    uint8_t* d_mask = nullptr;
    size_t smem = 0;
    int nt = 128;                  // threads per walker CTA
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    std::vector<double> h_inv_mass;
    std::vector<double> h_w, h_el, h_ids, h_par, h_nacc, h_ncut;
    double* h_stage = nullptr;     // pinned staging for the per-step scalar planes [8 * capacity]
    double next_id = 1.0;
    uint64_t h2d = 0, d2h = 0;     // bytes copied host->device / device->host
    uint64_t launches = 0;         // kernels launched by this context
    double* noalloc_scratch = nullptr;   // device address of g_noalloc_scratch on `device`
    const std::atomic<int>* cancel = nullptr;   // a server's cancel flag, read between steps
    alea_gpu::EstimatorSet* est = nullptr;      // observable estimators (alea_gpu_add_estimator)
    uint64_t fingerprint = 0;      // FNV-1a of the system's layout and tables (equal systems, equal records)
    std::vector<int> last_src;     // the last branch's map: new walker j copies old walker last_src[j]
    std::vector<DevOpt> h_opt;     // optimisable parameters of the pair terms (device pointers patched)
    DevOpt* d_opt = nullptr;
    double* d_opt_out = nullptr;   // [n_opt][capacity]
    double* d_opt_grad = nullptr;  // [n_opt][np*2][capacity] x 2 (gradient, Laplacian)
    double* d_opt_scratch = nullptr;   // Gaussian-width derivatives: 3 maxN^2 per CTA
    int orbital_opts = 0;          // kind-1 (Gaussian width) parameters among h_opt
    FwState* fw = nullptr;         // forward walking (alea_gpu_set_forward_walking)
    alea_gpu_checkpoint_fn ckpt_fn = nullptr;   // DMC milestone hook and its argument
    void* ckpt_user = nullptr;
    int prop_p = -1;               // alea_gpu_propose: the proposed particle and its positions [dim*nw]
    std::vector<double> prop_pos;
    DevSys* d_sys = nullptr;       // device copy of sys for packed launches (alea_gpu_vmc_run_packed)
};

namespace {

// NVTX range over one entry point's work (the phases of a step: sweep,
// branch, estimators, uploads), visible to ncu's --nvtx filters and any
// NVTX-aware tracer; no cost without one attached.
struct Phase {
    explicit Phase(const char* name) { nvtxRangePushA(name); }
    ~Phase() { nvtxRangePop(); }
    Phase(const Phase&) = delete;
    Phase& operator=(const Phase&) = delete;
};

int fail(alea_gpu_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    else g_create_error = msg;
    return code;
}

#define CUDA_TRY(ctx, expr)                                                               \
    do {                                                                                  \
        cudaError_t e_ = (expr);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail((ctx), ALEA_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

long round4(long x) { return (x + 3) & ~3L; }

// Pinned host staging blocks, reused across contexts for the life of the
// process: freeing pinned memory can synchronise the device, which would make
// a finishing context wait for the others' work.
std::mutex g_pinned_mu;
std::multimap<size_t, void*> g_pinned_free;

void* pinned_acquire(size_t bytes) {
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        auto it = g_pinned_free.lower_bound(bytes);
        if (it != g_pinned_free.end()) {
            void* p = it->second;
            g_pinned_free.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    // round up so that blocks are reusable by contexts of similar size
    size_t b = 1u << 16;
    while (b < bytes) b <<= 1;
    if (cudaMallocHost(&p, b) != cudaSuccess) return nullptr;
    return p;
}

void pinned_release(void* p, size_t bytes) {
    if (!p) return;
    size_t b = 1u << 16;
    while (b < bytes) b <<= 1;
    std::lock_guard<std::mutex> lk(g_pinned_mu);
    g_pinned_free.emplace(b, p);
}

// The device's default memory pool keeps what contexts free (no release at
// synchronisation points), so the next context's allocations are served from
// it.  A setting of this process's runtime, not of the GPU.
void keep_pool_warm(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    done[device] = true;
}

// e^x K0(x), e^x K1(x) on the host: the ascending series for x <= 2 (DLMF
// 10.31.1-2), the standard library's K_nu times e^x up to x = 30, and the
// Hankel asymptotic series e^x K_nu(x) = sqrt(π/2x) Σ a_k(ν)/x^k beyond
// (a_k = a_{k-1} (4ν² - (2k-1)²)/(8k); DLMF 10.40.2), summed to 1e-17.
void host_k01e(double x, double& k0e, double& k1e) {
    if (x <= 2.0) {
        const double euler_gamma = 0.57721566490153286060651209008240243;
        const double y = 0.25 * x * x;
        double term0 = 1.0, term1 = 1.0, harmonic = 0.0, i0 = 0.0, s0 = 0.0, i1 = 0.0, s1 = 0.0;
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
        const double lh = std::log(0.5 * x);
        const double ex = std::exp(x);
        k0e = ex * (-(lh + euler_gamma) * i0 + s0);
        k1e = ex * (1.0 / x + lh * (0.5 * x * i1) - 0.25 * x * s1);
        return;
    }
    if (x <= 30.0) {
        const double ex = std::exp(x);
        k0e = ex * std::cyl_bessel_k(0.0, x);
        k1e = ex * std::cyl_bessel_k(1.0, x);
        return;
    }
    const double pre = std::sqrt(3.14159265358979323846 / (2.0 * x));
    for (int nu = 0; nu < 2; ++nu) {
        const double mu = 4.0 * nu * nu;
        double a = 1.0, sum = 1.0;
        for (int k = 1; k < 60; ++k) {
            a *= (mu - (2.0 * k - 1) * (2.0 * k - 1)) / (8.0 * k * x);
            sum += a;
            if (std::abs(a) < 1e-17 * std::abs(sum)) break;
        }
        (nu == 0 ? k0e : k1e) = pre * sum;
    }
}

// Chebyshev coefficients of sqrt(x) e^x K_nu(x) in ξ = 4/x - 1 for ν = 0, 1
// (24 each), projected on 192 first-kind nodes ξ_j = cos θ_j.
std::vector<double> bessel_k01_chebyshev() {
    constexpr int kTerms = 24, M = 8 * kTerms;
    std::vector<double> f0(M), f1(M), theta(M), c(2 * kTerms, 0.0);
    for (int j = 0; j < M; ++j) {
        theta[j] = 3.14159265358979323846 * (j + 0.5) / M;
        const double x = 4.0 / (std::cos(theta[j]) + 1.0);
        double k0e, k1e;
        host_k01e(x, k0e, k1e);
        f0[j] = std::sqrt(x) * k0e;
        f1[j] = std::sqrt(x) * k1e;
    }
    for (int k = 0; k < kTerms; ++k) {
        double s0 = 0.0, s1 = 0.0;
        for (int j = 0; j < M; ++j) {
            const double ck = std::cos(k * theta[j]);
            s0 += f0[j] * ck;
            s1 += f1[j] * ck;
        }
        const double norm = (k == 0 ? 1.0 : 2.0) / M;
        c[k] = norm * s0;
        c[kTerms + k] = norm * s1;
    }
    return c;
}

// Per-interval monomial coefficients of a quintic Hermite spline: on interval
// i, with y = 1 − x,
//   f = a0 h0(x) + a1 h1(x) + a2 h2(x) + b0 h0(y) − b1 h1(y) + b2 h2(y),
//   h0 = 1 − 10x³ + 15x⁴ − 6x⁵, h1 = x − 6x³ + 8x⁴ − 3x⁵,
//   h2 = x²/2 − 3x³/2 + 3x⁴/2 − x⁵/2,
// (a, b the scaled data of knots i, i+1) expanded into c_0 + ... + c_5 x^5.
std::vector<double> hermite_to_monomial(const double* scaled, int n_knots) {
    static const double H[3][6] = {{1, 0, 0, -10, 15, -6}, {0, 1, 0, -6, 8, -3}, {0, 0, 0.5, -1.5, 1.5, -0.5}};
    // h_j(1 − x) in monomials of x
    double G[3][6] = {};
    for (int j = 0; j < 3; ++j)
        for (int m = 0; m < 6; ++m) {
            double binom = 1.0;   // C(m, q) (−1)^q
            for (int q = 0; q <= m; ++q) {
                G[j][q] += H[j][m] * binom;
                binom = -binom * (m - q) / (q + 1);
            }
        }
    std::vector<double> out(6 * static_cast<size_t>(std::max(n_knots - 1, 1)), 0.0);
    for (int i = 0; i + 1 < n_knots; ++i) {
        const double* a = scaled + 3 * i;
        const double* b = a + 3;
        for (int q = 0; q < 6; ++q)
            out[6 * i + q] = a[0] * H[0][q] + a[1] * H[1][q] + a[2] * H[2][q] + b[0] * G[0][q] -
                             b[1] * G[1][q] + b[2] * G[2][q];
    }
    return out;
}

// Host<->device copies on the context's stream, counted.
cudaError_t copy_in(alea_gpu_ctx* c, void* dst, const void* src, size_t n) {
    c->h2d += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, c->stream);
}
cudaError_t copy_out(alea_gpu_ctx* c, void* dst, const void* src, size_t n) {
    c->d2h += n;
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, c->stream);
}

// Threads per walker CTA: one warp while a move has at most a few tens of
// independent items (orbitals, partners, k vectors), wider for larger systems.
// ALEA_GPU_THREADS overrides (32, 64 or 128).
int pick_threads(const DevSys& s) {
    if (const char* e = std::getenv("ALEA_GPU_THREADS")) {
        const int v = std::atoi(e);
        if (v == 32 || v == 64 || v == 128) return v;
    }
    if (s.maxN <= 32 && s.np <= 64) return 32;
    if (s.maxN <= 48 && s.np <= 128) return 64;
    return 128;
}


// Cell from the lattice rows: axis alignment, 2-D Gauss reduction, (Aᵀ)⁻¹,
// the orthorhombic fold, the 3×3 candidate shell, reciprocal vectors.
int setup_cell(alea_gpu_ctx* c, const alea_gpu_system* in, DevSys& s) {
    s.periodic = in->periodic;
    s.ortho = 0;
    if (!s.periodic) return ALEA_OK;
    double a[4] = {in->lattice[0], in->lattice[1], in->lattice[2], in->lattice[3]};
    // axis_align
    int axis[2], used[2] = {0, 0};
    bool aligned = true;
    for (int i = 0; i < 2 && aligned; ++i) {
        int nz = 0, which = 0;
        for (int d = 0; d < 2; ++d)
            if (a[i * 2 + d] != 0.0) {
                ++nz;
                which = d;
            }
        if (nz != 1 || used[which]) aligned = false;
        else {
            axis[i] = which;
            used[which] = 1;
        }
    }
    if (aligned) {
        double r[4] = {0, 0, 0, 0};
        for (int i = 0; i < 2; ++i)
            for (int d = 0; d < 2; ++d) r[axis[i] * 2 + d] = a[i * 2 + d];
        std::memcpy(a, r, sizeof a);
        s.ortho = 1;
    } else {
        for (int guard = 0; guard < 64; ++guard) {
            const double n0 = a[0] * a[0] + a[1] * a[1], n1 = a[2] * a[2] + a[3] * a[3];
            if (n1 < n0) {
                std::swap(a[0], a[2]);
                std::swap(a[1], a[3]);
                continue;
            }
            if (n0 == 0.0) break;
            const double mu = std::nearbyint((a[0] * a[2] + a[1] * a[3]) / n0);
            if (mu == 0.0) break;
            a[2] -= mu * a[0];
            a[3] -= mu * a[1];
        }
    }
    const double det = a[0] * a[3] - a[1] * a[2];
    if (det == 0.0) return fail(c, ALEA_ERR_INVALID, "lattice vectors are singular");
    const double inv_det = 1.0 / det;
    std::memcpy(s.a, a, sizeof a);
    s.ainv[0] = a[3] * inv_det;
    s.ainv[1] = -a[2] * inv_det;
    s.ainv[2] = -a[1] * inv_det;
    s.ainv[3] = a[0] * inv_det;
    const double two_pi = 6.283185307179586476925286766559;
    for (int k = 0; k < 4; ++k) s.recip[k] = two_pi * s.ainv[k];
    if (s.ortho)
        for (int d = 0; d < 2; ++d) {
            s.box[d] = std::abs(a[d * 2 + d]);
            s.inv_box[d] = 1.0 / s.box[d];
        }
    int nc = 1;
    s.cand[0] = s.cand[1] = 0.0;
    if (!s.ortho)
        for (int n0 = -1; n0 <= 1; ++n0)
            for (int n1 = -1; n1 <= 1; ++n1) {
                if (n0 == 0 && n1 == 0) continue;
                for (int d = 0; d < 2; ++d) {
                    double acc = 0.0;
                    acc += n0 * a[0 * 2 + d];
                    acc += n1 * a[1 * 2 + d];
                    s.cand[nc * 2 + d] = acc;
                }
                ++nc;
            }
    return ALEA_OK;
}

// Host arena of tables, uploaded once; pointers are patched after cudaMalloc.
struct Arena {
    std::vector<char> bytes;
    size_t add(const void* p, size_t n) {
        const size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + n);
        if (n) std::memcpy(bytes.data() + off, p, n);
        return off;
    }
};

int build_system3(alea_gpu_ctx* c, const alea_gpu_system* in);

int build_system(alea_gpu_ctx* c, const alea_gpu_system* in) {
    DevSys& s = c->sys;
    s = DevSys{};
    if (!in) return fail(c, ALEA_ERR_INVALID, "null system");
    if (in->dim == 3) return build_system3(c, in);
    if (in->dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "the walker kernels implement dim = 2 and dim = 3");
    const int np = in->n_particles;
    if (np < 1 || np > 1024) return fail(c, ALEA_ERR_INVALID, "n_particles must be in [1, 1024]");
    s.dim = 2;
    s.np = np;
    if (int rc = setup_cell(c, in, s)) return rc;
    Arena ar;
    struct Patch { size_t off; const void** slot; };
    std::vector<Patch> patches;
    auto put = [&](const void* p, size_t n, const void** slot) {
        patches.push_back({ar.add(p, n), slot});
    };
    std::vector<std::vector<double>> poly_tables;
    std::vector<double> bessel_table;     // zero-energy terms' Chebyshev table (one per system)
    const double* bessel_dev = nullptr;   // patched to its device address
    std::vector<int> ze_terms;
    std::vector<double> bf_sin[2];
    // groups
    if (in->n_groups < 1 || in->n_groups > kMaxGroups) return fail(c, ALEA_ERR_INVALID, "bad n_groups");
    s.ngroups = in->n_groups;
    std::vector<double> inv_mass(np * 2, 0.0), charge(np, 0.0);
    std::vector<int> group_of(np, -1);
    for (int g = 0; g < in->n_groups; ++g) {
        const alea_gpu_group& G = in->groups[g];
        if (G.first < 0 || G.last > np || G.first >= G.last)
            return fail(c, ALEA_ERR_INVALID, "group range out of bounds");
        s.gfirst[g] = G.first;
        s.glast[g] = G.last;
        s.gcharge[g] = G.charge;
        for (int i = G.first; i < G.last; ++i) {
            if (group_of[i] >= 0) return fail(c, ALEA_ERR_INVALID, "groups overlap");
            group_of[i] = g;
            charge[i] = G.charge;
            inv_mass[i * 2] = G.inv_mass[0];
            inv_mass[i * 2 + 1] = G.inv_mass[1];
        }
    }
    for (int i = 0; i < np; ++i)
        if (group_of[i] < 0) return fail(c, ALEA_ERR_INVALID, "a particle belongs to no group");
    c->h_inv_mass = inv_mass;
    put(inv_mass.data(), inv_mass.size() * 8, reinterpret_cast<const void**>(&s.inv_mass));
    put(charge.data(), charge.size() * 8, reinterpret_cast<const void**>(&s.charge));
    put(group_of.data(), group_of.size() * 4, reinterpret_cast<const void**>(&s.group_of));

    // record layout, hot part
    long o = 0;
    s.o_pos = o; o += np * 2;
    s.o_jg = o; o += np * 2;
    s.o_jl = o; o += np * 2;
    s.o_kg = o; o += np * 2;
    s.o_kl = o; o += np * 2;
    s.o_sg = o; o += np * 2;
    s.o_sl = o; o += np * 2;
    s.o_scal = o; o += S_NSCAL;
    // a complex determinant is all twisted plane-wave blocks
    s.cplx = 0;
    for (int b = 0; b < in->n_blocks; ++b) s.cplx |= in->blocks[b].type == ALEA_ORB_TWISTED_PLANE_WAVE;
    if (s.cplx)
        for (int b = 0; b < in->n_blocks; ++b)
            if (in->blocks[b].type != ALEA_ORB_TWISTED_PLANE_WAVE)
                return fail(c, ALEA_ERR_UNSUPPORTED, "twisted plane-wave blocks cannot be mixed with real ones");
    s.o_pg = static_cast<int>(o); o += s.cplx ? np * 2 : 0;
    s.o_pl = static_cast<int>(o); o += s.cplx ? np * 2 : 0;
    // determinant blocks
    if (in->n_blocks < 0 || in->n_blocks > kMaxBlocks) return fail(c, ALEA_ERR_INVALID, "bad n_blocks");
    s.nblocks = in->n_blocks;
    s.maxN = 1;
    std::vector<std::vector<double>> sin_flags(in->n_blocks);
    for (int b = 0; b < in->n_blocks; ++b) {
        const alea_gpu_orbitals& B = in->blocks[b];
        DevBlock& D = s.blocks[b];
        D.first = B.first;
        D.last = B.last;
        D.n = B.last - B.first;
        D.type = B.type;
        if (D.n < 1 || D.n > kMaxN || B.first < 0 || B.last > np)
            return fail(c, ALEA_ERR_UNSUPPORTED, "determinant blocks must have 1..64 particles");
        s.maxN = std::max(s.maxN, D.n);
        if (B.type == ALEA_ORB_PLANE_WAVE) {
            if (!B.k || !B.is_sin) return fail(c, ALEA_ERR_INVALID, "plane-wave block without tables");
            put(B.k, D.n * 2 * 8, reinterpret_cast<const void**>(&D.k));
            sin_flags[b].resize(D.n);
            for (int i = 0; i < D.n; ++i) sin_flags[b][i] = B.is_sin[i] ? 1.0 : 0.0;
            put(sin_flags[b].data(), D.n * 8, reinterpret_cast<const void**>(&D.is_sin));
        } else if (B.type == ALEA_ORB_TWISTED_PLANE_WAVE) {
            if (!B.k) return fail(c, ALEA_ERR_INVALID, "twisted plane-wave block without wavevectors");
            put(B.k, D.n * 2 * 8, reinterpret_cast<const void**>(&D.k));
        } else if (B.type == ALEA_ORB_GAUSSIAN) {
            if (!B.centers || !B.alphas) return fail(c, ALEA_ERR_INVALID, "Gaussian block without tables");
            put(B.centers, D.n * 2 * 8, reinterpret_cast<const void**>(&D.centers));
            put(B.alphas, D.n * 8, reinterpret_cast<const void**>(&D.alphas));
        } else {
            return fail(c, ALEA_ERR_INVALID, "unknown orbital type");
        }
        D.oA = static_cast<int>(o);
        o += (s.cplx ? 2 : 1) * round4(D.n * D.n);
    }
    for (int b = 0; b < s.nblocks; ++b) {
        s.blocks[b].orabs = static_cast<int>(o);
        o += round4(s.blocks[b].n);
    }
    // backflow determinants (BackflowSlaterDeterminant): x, A = M⁻¹, F, (log|det|, sign)
    if (in->n_backflow < 0 || in->n_backflow > 2) return fail(c, ALEA_ERR_INVALID, "bad n_backflow");
    s.nbf = in->n_backflow;
    if (s.nbf > 0 && s.nblocks > 0)
        return fail(c, ALEA_ERR_UNSUPPORTED, "backflow determinants cannot be mixed with plain blocks");
    if (s.nbf > 0 && np > 256) return fail(c, ALEA_ERR_UNSUPPORTED, "backflow needs at most 256 particles");
    for (int d = 0; d < s.nbf; ++d) {
        const alea_gpu_backflow& F = in->backflow[d];
        DevBF& D = s.bf[d];
        D.first = F.first;
        D.last = F.last;
        D.n = F.last - F.first;
        D.type = F.type;
        if (D.n < 1 || D.n > kMaxN || F.first < 0 || F.last > np)
            return fail(c, ALEA_ERR_UNSUPPORTED, "backflow determinants must have 1..64 rows");
        s.maxN = std::max(s.maxN, D.n);
        if (F.type == ALEA_ORB_PLANE_WAVE) {
            if (!F.k || !F.is_sin) return fail(c, ALEA_ERR_INVALID, "backflow plane waves without tables");
            put(F.k, D.n * 2 * 8, reinterpret_cast<const void**>(&D.k));
            bf_sin[d].resize(D.n);
            for (int i = 0; i < D.n; ++i) bf_sin[d][i] = F.is_sin[i] ? 1.0 : 0.0;
            put(bf_sin[d].data(), D.n * 8, reinterpret_cast<const void**>(&D.is_sin));
        } else if (F.type == ALEA_ORB_GAUSSIAN) {
            if (!F.centers || !F.alphas) return fail(c, ALEA_ERR_INVALID, "backflow Gaussians without tables");
            put(F.centers, D.n * 2 * 8, reinterpret_cast<const void**>(&D.centers));
            put(F.alphas, D.n * 8, reinterpret_cast<const void**>(&D.alphas));
        } else {
            return fail(c, ALEA_ERR_UNSUPPORTED, "backflow orbitals must be plane waves or Gaussians");
        }
        if (F.n_channels < 1 || F.n_channels > 4) return fail(c, ALEA_ERR_INVALID, "bad backflow channels");
        D.nch = F.n_channels;
        for (int q = 0; q < D.nch; ++q) {
            const alea_gpu_backflow_channel& C = F.channels[q];
            DevBFCh& E = D.ch[q];
            if (C.source_first < 0 || C.source_last > np || C.source_first >= C.source_last || C.C < 2 ||
                !(C.L > 0.0) || C.n_coeffs < 1 || C.n_coeffs > 16)
                return fail(c, ALEA_ERR_INVALID, "bad backflow channel");
            E.sf = C.source_first;
            E.sl = C.source_last;
            E.C = C.C;
            E.L = C.L;
            E.nc = C.n_coeffs;
            for (int k = 0; k < E.nc; ++k) E.c[k] = C.coeffs[k];
        }
        D.oX = static_cast<int>(o); o += round4(2 * D.n);
        D.oA = static_cast<int>(o); o += round4(D.n * D.n);
        D.oF = static_cast<int>(o); o += round4(2 * D.n);
        D.oLS = static_cast<int>(o); o += 4;
    }
    // pair terms and the shared Jastrow k set
    if (in->n_terms < 0 || in->n_terms > kMaxTerms) return fail(c, ALEA_ERR_INVALID, "bad n_terms");
    s.nterms = in->n_terms;
    const alea_gpu_kset* kref = nullptr;
    std::vector<double> kx2, ky2;
    for (int t = 0; t < in->n_terms; ++t) {
        const alea_gpu_pair_term& T = in->terms[t];
        DevTerm& D = s.terms[t];
        D.kind = T.kind;
        D.npairs = T.n_pairs;
        if (T.n_pairs < 1 || T.n_pairs > ALEA_GPU_MAX_PAIRS) return fail(c, ALEA_ERR_INVALID, "bad n_pairs");
        for (int q = 0; q < T.n_pairs; ++q)
            for (int k = 0; k < 4; ++k) {
                D.pairs[q][k] = T.pairs[q][k];
                if (T.pairs[q][k] < 0 || T.pairs[q][k] > np)
                    return fail(c, ALEA_ERR_INVALID, "pair range out of bounds");
            }
        D.same0 = T.pairs[0][0] == T.pairs[0][2] && T.pairs[0][1] == T.pairs[0][3];
        if (T.kind == ALEA_PAIR_PADE) {
            if (T.n_pairs != 1) return fail(c, ALEA_ERR_INVALID, "a Padé term has one group pair");
            if (T.num_order + T.den_order > 16 || T.num_order < 0 || T.den_order < 0)
                return fail(c, ALEA_ERR_INVALID, "Padé order too large");
            D.nnum = T.num_order;
            D.nden = T.den_order;
            for (int k = 0; k < D.nnum + D.nden; ++k) D.coef[k] = T.coeffs[k];
            D.image = T.image_sum;
            if (T.image_sum) {
                if (!s.periodic) return fail(c, ALEA_ERR_INVALID, "image sum in an open cell");
                const alea_gpu_spline& sp = T.short_range;
                if (!sp.scaled || sp.n_knots < 2) return fail(c, ALEA_ERR_INVALID, "bad image-sum spline");
                D.sp.r_cut = sp.r_cut;
                D.sp.inv_delta = sp.inv_delta;
                D.sp.n_knots = sp.n_knots;
                put(sp.scaled, 3 * sp.n_knots * 8, reinterpret_cast<const void**>(&D.sp.scaled));
                poly_tables.push_back(hermite_to_monomial(sp.scaled, sp.n_knots));
                put(poly_tables.back().data(), poly_tables.back().size() * 8,
                    reinterpret_cast<const void**>(&D.sp.poly));
                D.u_inf = T.u_inf;
                const alea_gpu_kset& ks = T.kset;
                if (ks.n_k < 1 || !ks.n1 || !ks.n2 || !ks.kx || !ks.ky || !ks.weight)
                    return fail(c, ALEA_ERR_INVALID, "bad image-sum k set");
                if (!kref) {
                    kref = &ks;
                } else if (ks.n_k != kref->n_k || std::memcmp(ks.n1, kref->n1, 4 * ks.n_k) ||
                           std::memcmp(ks.n2, kref->n2, 4 * ks.n_k)) {
                    return fail(c, ALEA_ERR_UNSUPPORTED, "image-summed terms must share one k set");
                }
                put(ks.weight, ks.n_k * 8, reinterpret_cast<const void**>(&D.kw));
                // the structure factor is kept per particle group
                for (int side = 0; side < 2; ++side) {
                    const int f0 = T.pairs[0][side * 2], f1 = T.pairs[0][side * 2 + 1];
                    bool ok = false;
                    for (int g = 0; g < s.ngroups; ++g) ok |= s.gfirst[g] == f0 && s.glast[g] == f1;
                    if (!ok) return fail(c, ALEA_ERR_UNSUPPORTED, "image-summed term on a partial group");
                }
            }
        } else if (T.kind == ALEA_PAIR_DRUMMOND) {
            if (T.C < 2 || T.n_coeffs < 1 || T.n_coeffs > 16) return fail(c, ALEA_ERR_INVALID, "bad Drummond term");
            D.C = T.C;
            D.gamma = T.gamma;
            D.L = T.L;
            D.ncoef = T.n_coeffs;
            for (int k = 0; k < T.n_coeffs; ++k) D.dc[k] = T.dcoeffs[k];
            double ipw = 1.0;
            for (int i = 0; i < T.C; ++i) ipw *= -T.L;
            D.alpha1 = T.gamma / ipw + D.dc[0] * static_cast<double>(T.C) / T.L;
        } else if (T.kind == ALEA_PAIR_ZERO_ENERGY) {
            // ZeroEnergyFunction (src/wavefunction/zero_energy_jastrow.cpp:16-60)
            if (T.n_pairs != 1) return fail(c, ALEA_ERR_INVALID, "a zero-energy term has one group pair");
            const double b = T.ze_b, p = T.ze_exponent, rm = T.ze_matching_radius, rc = T.ze_cutoff;
            if (!(std::isfinite(b) && b > 0.0) || !(std::isfinite(p) && p > 2.0) ||
                !(std::isfinite(rc) && rc > 0.0) || !(rm > 0.0 && rm < rc))
                return fail(c, ALEA_ERR_INVALID,
                            "zero-energy term needs b > 0, exponent > 2 and 0 < matching radius < cutoff");
            if (bessel_table.empty()) {
                bessel_table = bessel_k01_chebyshev();
                put(bessel_table.data(), bessel_table.size() * 8, reinterpret_cast<const void**>(&bessel_dev));
            }
            D.ze_s = 0.5 * (p - 2.0);
            D.ze_kappa = std::sqrt(b) / D.ze_s;
            D.ze_rm = rm;
            D.ze_rc = rc;
            const double x = D.ze_kappa * std::pow(rm, -D.ze_s);
            double k0e, k1e;
            host_k01e(x, k0e, k1e);
            const double q = k1e / k0e, sx = D.ze_s * x;
            const double u0 = std::log(k0e) - x, du0 = sx * q / rm;
            const double cc = 2.0 * rc - rm;
            const double h = 1.0 / (rm * rm) - 1.0 / (cc * cc);
            D.ze_c3 = du0 / h;
            D.ze_logc2 = 2.0 * D.ze_c3 / rc;
            D.ze_logc1 = D.ze_logc2 - D.ze_c3 / rm - D.ze_c3 / cc - u0;
            ze_terms.push_back(t);
        } else {
            return fail(c, ALEA_ERR_INVALID, "unknown pair term");
        }
    }
    // optimisable parameters of the pair terms (alea_gpu_parameter_derivatives)
    c->h_opt.clear();
    c->h_opt.reserve(static_cast<size_t>(kMaxTerms + 8) * ALEA_GPU_MAX_OPT + kMaxBlocks);
    for (int b = 0; b < in->n_blocks; ++b) {
        const alea_gpu_orbitals& O = in->blocks[b];
        if (!O.opt_alpha) continue;
        const int n = O.last - O.first;
        bool uniform = O.type == ALEA_ORB_GAUSSIAN && n > 0;
        for (int i = 1; uniform && i < n; ++i) uniform = O.alphas[i] == O.alphas[0];
        if (!uniform)
            return fail(c, ALEA_ERR_INVALID, "opt_alpha needs a Gaussian block of one shared width");
        c->h_opt.push_back(DevOpt{});
        c->h_opt.back().kind = 1;
        c->h_opt.back().term = b;
    }
    // backflow channels' parameters, BackflowFunction's order [c_0, (c_1), c_2.., L]
    // (backflow_function.h:111-135) mapped to a coefficient index or -1 for L
    for (int d = 0; d < in->n_backflow; ++d)
        for (int q = 0; q < in->backflow[d].n_channels; ++q) {
            const alea_gpu_backflow_channel& C = in->backflow[d].channels[q];
            const int zs = C.zero_slope ? 1 : 0;
            if (C.n_opt < 0 || C.n_opt > ALEA_GPU_MAX_OPT || (zs && C.n_coeffs < 2))
                return fail(c, ALEA_ERR_INVALID, "bad backflow n_opt / zero_slope");
            const int n_par = C.n_coeffs - zs + 1;
            for (int u = 0; u < C.n_opt; ++u) {
                const int slot = C.opt_index[u];
                if (slot < 0 || slot >= n_par || (u > 0 && slot <= C.opt_index[u - 1]))
                    return fail(c, ALEA_ERR_INVALID, "backflow opt_index out of range or not ascending");
                c->h_opt.push_back(DevOpt{});
                DevOpt& o = c->h_opt.back();
                o.kind = 2;
                o.term = d;
                o.ch = q;
                o.zs = zs;
                o.index = slot == n_par - 1 ? -1 : (zs && slot >= 1 ? slot + 1 : slot);
            }
        }
    for (int t = 0; t < in->n_terms; ++t) {
        const alea_gpu_pair_term& T = in->terms[t];
        if (T.n_opt < 0 || T.n_opt > ALEA_GPU_MAX_OPT) return fail(c, ALEA_ERR_INVALID, "bad n_opt");
        if (T.n_opt > 0 && T.kind == ALEA_PAIR_ZERO_ENERGY)
            return fail(c, ALEA_ERR_UNSUPPORTED, "zero-energy terms have no optimisable parameters here");
        for (int q = 0; q < T.n_opt; ++q) {
            const int idx = T.opt_index[q];
            const int limit = T.kind == ALEA_PAIR_PADE ? T.num_order + T.den_order : T.n_coeffs + 1;
            if (idx < 0 || idx >= limit) return fail(c, ALEA_ERR_INVALID, "opt_index out of range");
            c->h_opt.push_back(DevOpt{});
            DevOpt& o = c->h_opt.back();
            o.term = t;
            o.index = idx;
            if (T.kind == ALEA_PAIR_PADE && T.image_sum) {
                const alea_gpu_spline& sp = T.opt_short_range[q];
                if (!sp.scaled || sp.n_knots < 2 || !T.opt_weight[q])
                    return fail(c, ALEA_ERR_INVALID, "an image-summed Padé parameter needs its breakup tables");
                o.inf = T.opt_inf[q];
                o.sp.r_cut = sp.r_cut;
                o.sp.inv_delta = sp.inv_delta;
                o.sp.n_knots = sp.n_knots;
                put(sp.scaled, 3 * sp.n_knots * 8, reinterpret_cast<const void**>(&o.sp.scaled));
                poly_tables.push_back(hermite_to_monomial(sp.scaled, sp.n_knots));
                put(poly_tables.back().data(), poly_tables.back().size() * 8,
                    reinterpret_cast<const void**>(&o.sp.poly));
                put(T.opt_weight[q], T.kset.n_k * 8, reinterpret_cast<const void**>(&o.kw));
            }
        }
    }
    // group-pair coupling masks, when every term's ranges are whole groups
    {
        auto group_at = [&](int f, int l) {
            for (int g = 0; g < s.ngroups; ++g)
                if (s.gfirst[g] == f && s.glast[g] == l) return g;
            return -1;
        };
        s.pair_by_group = 1;
        std::memset(s.gterms, 0, sizeof s.gterms);
        for (int t = 0; t < s.nterms; ++t)
            for (int q = 0; q < s.terms[t].npairs; ++q) {
                const int ga = group_at(s.terms[t].pairs[q][0], s.terms[t].pairs[q][1]);
                const int gb = group_at(s.terms[t].pairs[q][2], s.terms[t].pairs[q][3]);
                if (ga < 0 || gb < 0) {
                    s.pair_by_group = 0;
                    continue;
                }
                s.gterms[ga][gb] |= static_cast<uint8_t>(1u << t);
                s.gterms[gb][ga] |= static_cast<uint8_t>(1u << t);
            }
    }
    if (kref) {
        s.nkJ = kref->n_k;
        int m1 = 0, m2 = 0;
        for (int k = 0; k < kref->n_k; ++k) {
            m1 = std::max(m1, std::abs(kref->n1[k]));
            m2 = std::max(m2, std::abs(kref->n2[k]));
            kx2.push_back(kref->kx[k] * kref->kx[k]);
            ky2.push_back(kref->ky[k] * kref->ky[k]);
        }
        if (m1 > kMaxLadder || m2 > kMaxLadder) return fail(c, ALEA_ERR_UNSUPPORTED, "k index too large");
        s.m1J = m1;
        s.m2J = m2;
        put(kref->n1, 4 * s.nkJ, reinterpret_cast<const void**>(&s.n1J));
        put(kref->n2, 4 * s.nkJ, reinterpret_cast<const void**>(&s.n2J));
        put(kref->kx, 8 * s.nkJ, reinterpret_cast<const void**>(&s.kxJ));
        put(kref->ky, 8 * s.nkJ, reinterpret_cast<const void**>(&s.kyJ));
        put(kx2.data(), 8 * s.nkJ, reinterpret_cast<const void**>(&s.kx2J));
        put(ky2.data(), 8 * s.nkJ, reinterpret_cast<const void**>(&s.ky2J));
    }
    s.o_rho = static_cast<int>(o);
    o += static_cast<long>(s.ngroups) * 2 * s.nkJ;
    s.hot = static_cast<int>(round4(o));
    o = s.hot;
    for (int b = 0; b < s.nblocks; ++b) {   // twisted plane waves recompute their rows
        DevBlock& D = s.blocks[b];
        const long f = s.cplx ? 0 : 1;
        D.oD = o; o += f * round4(D.n * D.n);
        D.oDg = o; o += f * round4(D.n * D.n * 2);
        D.oDl = o; o += f * round4(D.n * D.n * 2);
    }
    s.rec = round4(o);
    // Ewald
    s.ewald = in->ewald.enabled;
    if (s.ewald) {
        const alea_gpu_ewald& E = in->ewald;
        if (!s.periodic) return fail(c, ALEA_ERR_INVALID, "Ewald in an open cell");
        if (!E.long_range.scaled || E.kset.n_k < 0 || (E.kset.n_k > 0 && (!E.kset.n1 || !E.kset.n2 || !E.kset.weight)))
            return fail(c, ALEA_ERR_INVALID, "bad Ewald tables");
        s.esp.r_cut = E.long_range.r_cut;
        s.esp.inv_delta = E.long_range.inv_delta;
        s.esp.n_knots = E.long_range.n_knots;
        put(E.long_range.scaled, 3 * E.long_range.n_knots * 8, reinterpret_cast<const void**>(&s.esp.scaled));
        poly_tables.push_back(hermite_to_monomial(E.long_range.scaled, E.long_range.n_knots));
        put(poly_tables.back().data(), poly_tables.back().size() * 8, reinterpret_cast<const void**>(&s.esp.poly));
        s.e_rcut = E.r_cut;
        s.e_inv_eps = E.inv_eps;
        s.e_const = E.constant;
        s.enk = E.kset.n_k;
        int m1 = 0, m2 = 0;
        for (int k = 0; k < s.enk; ++k) {
            m1 = std::max(m1, std::abs(E.kset.n1[k]));
            m2 = std::max(m2, std::abs(E.kset.n2[k]));
        }
        if (m1 > kMaxLadder || m2 > kMaxLadder) return fail(c, ALEA_ERR_UNSUPPORTED, "Ewald k index too large");
        s.e_m1 = m1;
        s.e_m2 = m2;
        if (s.enk > 0) {
            put(E.kset.n1, 4 * s.enk, reinterpret_cast<const void**>(&s.en1));
            put(E.kset.n2, 4 * s.enk, reinterpret_cast<const void**>(&s.en2));
            put(E.kset.weight, 8 * s.enk, reinterpret_cast<const void**>(&s.ew));
        }
    }
    if (in->n_coulomb < 0 || in->n_coulomb > kMaxCoulomb) return fail(c, ALEA_ERR_INVALID, "bad n_coulomb");
    s.ncoul = in->n_coulomb;
    for (int k = 0; k < s.ncoul; ++k) {
        const alea_gpu_coulomb& C = in->coulomb[k];
        s.coul[k][0] = C.a_first;
        s.coul[k][1] = C.a_last;
        s.coul[k][2] = C.b_first;
        s.coul[k][3] = C.b_last;
        s.coul_coef[k] = C.coef;
    }
    if (in->n_inverse_power < 0 || in->n_inverse_power > kMaxCoulomb)
        return fail(c, ALEA_ERR_INVALID, "bad n_inverse_power");
    s.nip = in->n_inverse_power;
    s.ip_tail = 0.0;
    for (int k = 0; k < s.nip; ++k) {
        const alea_gpu_inverse_power& V = in->inverse_power[k];
        if (V.a_first < 0 || V.a_last > np || V.b_first < 0 || V.b_last > np || V.a_first >= V.a_last ||
            V.b_first >= V.b_last || !(std::isfinite(V.exponent) && V.exponent > 0.0) ||
            !std::isfinite(V.strength))
            return fail(c, ALEA_ERR_INVALID, "bad inverse-power term");
        s.ip[k][0] = V.a_first;
        s.ip[k][1] = V.a_last;
        s.ip[k][2] = V.b_first;
        s.ip[k][3] = V.b_last;
        s.ip_c[k] = V.strength;
        s.ip_p[k] = V.exponent;
        const double rp = std::nearbyint(V.exponent);
        s.ip_pint[k] = (rp == V.exponent && rp <= 16.0) ? static_cast<int>(rp) : 0;
        s.ip_tail += V.tail;
    }
    // ziggurat tables
    const Ziggurat z = make_ziggurat();
    put(z.k, sizeof z.k, reinterpret_cast<const void**>(&s.zk));
    put(z.w, sizeof z.w, reinterpret_cast<const void**>(&s.zw));
    put(z.f, sizeof z.f, reinterpret_cast<const void**>(&s.zf));
    s.zr = z.r;
    // shared-memory layout after the hot part
    long m = s.hot;
    auto take = [&](long n) {
        const long at = m;
        m += round4(std::max(n, 1L));
        return static_cast<int>(at);
    };
    const long cf = s.cplx ? 2 : 1;   // complex rows and factors: re | im
    s.s_newpos = take(4);
    s.s_nval = take(cf * s.maxN);
    s.s_ngrad = take(2 * s.maxN);
    s.s_nlap = take(2 * s.maxN);
    s.s_cn = take(s.nkJ);
    s.s_sn = take(s.nkJ);
    s.s_co = take(s.nkJ);
    s.s_so = take(s.nkJ);
    s.s_col = take(cf * s.maxN);
    s.s_rowp = take(cf * s.maxN);
    s.s_red = take(4 * 16 + 16);
    s.s_misc = take(32 + 4 * 2 * (kMaxLadder + 1));
    // One union: the per-partner scratch of a move (read by the commit before
    // any rebuild), the Gauss-Jordan work matrix, and the ρ(k) accumulators
    // of the local energy.
    for (int d = 0; d < s.nbf; ++d) {   // a proposal's pending backflow state
        DevBF& D = s.bf[d];
        D.pX = take(2 * D.n);
        D.pA = take(D.n * D.n);
        D.pF = take(2 * D.n);
        D.pM = take(8);
    }
    long work = cf * s.maxN * s.maxN;
    // backflow: rows ∇φ (2N²) and G^α (2N²), T (4N), Jacobian columns (4N)
    for (int d = 0; d < s.nbf; ++d) work = std::max(work, 4L * s.bf[d].n * s.bf[d].n + 8L * s.bf[d].n);
    work = std::max(work, 2L * s.enk);
    work = std::max(work, static_cast<long>(np) * 10);
    work = std::max(work, 2L * s.ngroups * s.nkJ);   // one-warp k-space refresh: E_g(k)
    s.s_work = take(work);
    s.s_rad = s.s_work;
    s.s_total = static_cast<int>(m);
    c->smem = static_cast<size_t>(s.s_total) * 8;
    // the one-warp sweep's layout (see DevSys)
    s.f_total = 0;
    if (fast_sweep_eligible(s) || boson_sweep_eligible(s)) {
        const long np2 = 2L * np;
        long f = 0;
        auto ftake = [&](long n) {
            const long at = f;
            f += round4(std::max(n, 1L));
            return static_cast<int>(at);
        };
        s.f_pos = ftake(np2);
        s.f_jg = ftake(np2);
        s.f_jl = ftake(np2);
        s.f_scal = ftake(s.hot - s.o_scal);
        s.f_misc = ftake(8);   // the error flag lives through the whole sweep
        const long scratch = f;
        s.f_nval = ftake(cf * s.maxN);
        s.f_ngrad = ftake(2L * s.maxN);
        s.f_nlap = ftake(2L * s.maxN);
        s.f_col = ftake(cf * s.maxN);
        s.f_rowp = ftake(cf * s.maxN);
        s.f_work = static_cast<int>(f);
        // the move union: the partners' and phases' changes (the FP64 sweep
        // inverts in place); the FP32 form's FP64 rebuild also needs N² there
        const long changes = round4(4L * np) + 4 * round4(std::max(s.nkJ, 1));
        s.f_cn = s.f_work + static_cast<int>(round4(4L * np));
        s.f_sn = s.f_cn + static_cast<int>(round4(std::max(s.nkJ, 1)));
        s.f_co = s.f_sn + static_cast<int>(round4(std::max(s.nkJ, 1)));
        s.f_so = s.f_co + static_cast<int>(round4(std::max(s.nkJ, 1)));
        const long moves_end = f + changes;
        const long moves_end32 = f + std::max(round4(static_cast<long>(s.maxN) * s.maxN), changes);
        f = scratch;   // the local energy reuses the whole scratch area
        s.f_sg = ftake(np2);
        s.f_sl = ftake(np2);
        s.f_kg = ftake(np2);
        s.f_kl = ftake(np2);
        s.f_elwork = static_cast<int>(f);
        f += round4(std::max({2L * s.ngroups * s.nkJ, 2L * s.enk, 1L}));
        s.f_total = static_cast<int>(std::max(f, moves_end));
        s.f_total32 = static_cast<int>(std::max(f, moves_end32));
    }
    if (c->smem > 227 * 1024)
        return fail(c, ALEA_ERR_UNSUPPORTED,
                    "walker state needs " + std::to_string(c->smem) + " bytes of shared memory (> 227 KB)");
    // fingerprint before the pointers are patched: layout, scalars and tables
    {
        uint64_t h = 1469598103934665603ULL;
        auto mix = [&h](const void* p, size_t n) {
            const unsigned char* b = static_cast<const unsigned char*>(p);
            for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
        };
        mix(&s, sizeof s);
        mix(ar.bytes.data(), ar.bytes.size());
        c->fingerprint = h;
    }
    // upload the arena and patch pointers
    CUDA_TRY(c, cudaMallocAsync(&c->arena, std::max<size_t>(ar.bytes.size(), 256), c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->arena, ar.bytes.data(), ar.bytes.size(), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));   // ar.bytes is freed on return
    for (const Patch& p : patches) *p.slot = static_cast<char*>(c->arena) + p.off;
    for (int t : ze_terms) s.terms[t].ze_cheb = bessel_dev;
    c->orbital_opts = 0;
    for (const DevOpt& o : c->h_opt) c->orbital_opts += o.kind == 1;
    if (!c->h_opt.empty()) {
        CUDA_TRY(c, cudaMallocAsync(&c->d_opt, c->h_opt.size() * sizeof(DevOpt), c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->d_opt, c->h_opt.data(), c->h_opt.size() * sizeof(DevOpt),
                                    cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    return ALEA_OK;
}

// Three-dimensional systems, run by the walker kernels of alea_bf3d.cu: a
// periodic cell whose lattice rows lie along the axes (the orthorhombic fold)
// or an open one; backflow determinants, or plain determinants taken as
// backflow determinants without channels (plane waves or Gaussians, at most
// two); Drummond or minimum-image Padé pair terms; the 3-D Ewald sum (a k
// set with kz) and open Coulomb terms.  Every walker's state is hot.
int build_system3(alea_gpu_ctx* c, const alea_gpu_system* in) {
    DevSys& s = c->sys;
    const int np = in->n_particles;
    if (np < 1 || np > 256) return fail(c, ALEA_ERR_INVALID, "a three-dimensional system has 1..256 particles");
    s.dim = 3;
    s.np = np;
    s.periodic = in->periodic;
    s.ortho = 1;
    if (s.periodic) {
        for (int i = 0; i < 3; ++i)
            for (int d = 0; d < 3; ++d)
                if (i != d && in->lattice[i * 3 + d] != 0.0)
                    return fail(c, ALEA_ERR_UNSUPPORTED,
                                "three-dimensional cells must be orthorhombic with rows along the axes");
        for (int d = 0; d < 3; ++d) {
            s.box[d] = std::abs(in->lattice[d * 3 + d]);
            if (!(s.box[d] > 0.0) || !std::isfinite(s.box[d]))
                return fail(c, ALEA_ERR_INVALID, "lattice vectors are singular");
            s.inv_box[d] = 1.0 / s.box[d];
        }
    }
    Arena ar;
    struct Patch { size_t off; const void** slot; };
    std::vector<Patch> patches;
    auto put = [&](const void* p, size_t n, const void** slot) { patches.push_back({ar.add(p, n), slot}); };
    if (in->n_groups < 1 || in->n_groups > kMaxGroups) return fail(c, ALEA_ERR_INVALID, "bad n_groups");
    s.ngroups = in->n_groups;
    std::vector<double> inv_mass(np * 3, 0.0), charge(np, 0.0);
    std::vector<int> group_of(np, -1);
    for (int g = 0; g < in->n_groups; ++g) {
        const alea_gpu_group& G = in->groups[g];
        if (G.first < 0 || G.last > np || G.first >= G.last)
            return fail(c, ALEA_ERR_INVALID, "group range out of bounds");
        s.gfirst[g] = G.first;
        s.glast[g] = G.last;
        s.gcharge[g] = G.charge;
        for (int i = G.first; i < G.last; ++i) {
            if (group_of[i] >= 0) return fail(c, ALEA_ERR_INVALID, "groups overlap");
            group_of[i] = g;
            charge[i] = G.charge;
            for (int d = 0; d < 3; ++d) inv_mass[i * 3 + d] = G.inv_mass[d];
        }
    }
    for (int i = 0; i < np; ++i)
        if (group_of[i] < 0) return fail(c, ALEA_ERR_INVALID, "a particle belongs to no group");
    c->h_inv_mass = inv_mass;
    put(inv_mass.data(), inv_mass.size() * 8, reinterpret_cast<const void**>(&s.inv_mass));
    put(charge.data(), charge.size() * 8, reinterpret_cast<const void**>(&s.charge));
    put(group_of.data(), group_of.size() * 4, reinterpret_cast<const void**>(&s.group_of));
    long o = 0;
    s.o_pos = o; o += np * 3;
    s.o_jg = o; o += np * 3;
    s.o_jl = o; o += np * 3;
    s.o_kg = o; o += np * 3;
    s.o_kl = o; o += np * 3;
    s.o_sg = o; o += np * 3;
    s.o_sl = o; o += np * 3;
    s.o_scal = o; o += S_NSCAL;
    s.cplx = 0;
    s.o_pg = s.o_pl = static_cast<int>(o);
    s.nblocks = 0;
    if (in->n_blocks > 0 && in->n_backflow > 0)
        return fail(c, ALEA_ERR_UNSUPPORTED, "backflow determinants cannot be mixed with plain blocks");
    const int ndet = in->n_backflow > 0 ? in->n_backflow : in->n_blocks;
    if (ndet < 0 || ndet > 2) return fail(c, ALEA_ERR_UNSUPPORTED, "a three-dimensional system has at most two determinants");
    s.nbf = ndet;
    s.maxN = 1;
    std::vector<double> sin_flags[2];
    for (int d = 0; d < ndet; ++d) {
        DevBF& D = s.bf[d];
        const bool bf = in->n_backflow > 0;
        const alea_gpu_backflow* F = bf ? &in->backflow[d] : nullptr;
        const alea_gpu_orbitals* B = bf ? nullptr : &in->blocks[d];
        D.first = bf ? F->first : B->first;
        D.last = bf ? F->last : B->last;
        D.n = D.last - D.first;
        D.type = bf ? F->type : B->type;
        if (D.n < 1 || D.n > 32 || D.first < 0 || D.last > np)
            return fail(c, ALEA_ERR_UNSUPPORTED, "three-dimensional determinants must have 1..32 rows");
        s.maxN = std::max(s.maxN, D.n);
        const double* k = bf ? F->k : B->k;
        const int* is_sin = bf ? F->is_sin : B->is_sin;
        const double* centers = bf ? F->centers : B->centers;
        const double* alphas = bf ? F->alphas : B->alphas;
        if (D.type == ALEA_ORB_PLANE_WAVE) {
            if (!k || !is_sin) return fail(c, ALEA_ERR_INVALID, "plane-wave determinant without tables");
            put(k, D.n * 3 * 8, reinterpret_cast<const void**>(&D.k));
            sin_flags[d].resize(D.n);
            for (int i = 0; i < D.n; ++i) sin_flags[d][i] = is_sin[i] ? 1.0 : 0.0;
            put(sin_flags[d].data(), D.n * 8, reinterpret_cast<const void**>(&D.is_sin));
        } else if (D.type == ALEA_ORB_GAUSSIAN) {
            if (!centers || !alphas) return fail(c, ALEA_ERR_INVALID, "Gaussian determinant without tables");
            put(centers, D.n * 3 * 8, reinterpret_cast<const void**>(&D.centers));
            put(alphas, D.n * 8, reinterpret_cast<const void**>(&D.alphas));
        } else {
            return fail(c, ALEA_ERR_UNSUPPORTED, "three-dimensional orbitals must be plane waves or Gaussians");
        }
        D.nch = 0;
        if (bf) {
            if (F->n_channels < 1 || F->n_channels > 4) return fail(c, ALEA_ERR_INVALID, "bad backflow channels");
            D.nch = F->n_channels;
            for (int q = 0; q < D.nch; ++q) {
                const alea_gpu_backflow_channel& C = F->channels[q];
                DevBFCh& E = D.ch[q];
                if (C.source_first < 0 || C.source_last > np || C.source_first >= C.source_last || C.C < 2 ||
                    !(C.L > 0.0) || C.n_coeffs < 1 || C.n_coeffs > 16)
                    return fail(c, ALEA_ERR_INVALID, "bad backflow channel");
                if (s.periodic && C.L > 0.5 * std::min({s.box[0], s.box[1], s.box[2]}))
                    return fail(c, ALEA_ERR_INVALID, "a backflow cutoff exceeds half the cell");
                E.sf = C.source_first;
                E.sl = C.source_last;
                E.C = C.C;
                E.L = C.L;
                E.nc = C.n_coeffs;
                for (int q2 = 0; q2 < E.nc; ++q2) E.c[q2] = C.coeffs[q2];
            }
        }
        D.oX = static_cast<int>(o); o += round4(3 * D.n);
        D.oA = static_cast<int>(o); o += round4(D.n * D.n);
        D.oF = static_cast<int>(o); o += round4(3 * D.n);
        D.oLS = static_cast<int>(o); o += 4;
    }
    if (in->n_terms < 0 || in->n_terms > kMaxTerms) return fail(c, ALEA_ERR_INVALID, "bad n_terms");
    s.nterms = in->n_terms;
    for (int t = 0; t < in->n_terms; ++t) {
        const alea_gpu_pair_term& T = in->terms[t];
        DevTerm& D = s.terms[t];
        D.kind = T.kind;
        D.npairs = T.n_pairs;
        if (T.n_pairs < 1 || T.n_pairs > ALEA_GPU_MAX_PAIRS) return fail(c, ALEA_ERR_INVALID, "bad n_pairs");
        for (int q = 0; q < T.n_pairs; ++q)
            for (int k = 0; k < 4; ++k) {
                D.pairs[q][k] = T.pairs[q][k];
                if (T.pairs[q][k] < 0 || T.pairs[q][k] > np)
                    return fail(c, ALEA_ERR_INVALID, "pair range out of bounds");
            }
        D.same0 = T.pairs[0][0] == T.pairs[0][2] && T.pairs[0][1] == T.pairs[0][3];
        if (T.kind == ALEA_PAIR_PADE) {
            if (T.image_sum) return fail(c, ALEA_ERR_UNSUPPORTED, "three-dimensional Padé terms are minimum-image only");
            if (T.num_order + T.den_order > 16 || T.num_order < 0 || T.den_order < 0)
                return fail(c, ALEA_ERR_INVALID, "Padé order too large");
            D.nnum = T.num_order;
            D.nden = T.den_order;
            for (int k = 0; k < D.nnum + D.nden; ++k) D.coef[k] = T.coeffs[k];
            D.image = 0;
        } else if (T.kind == ALEA_PAIR_DRUMMOND) {
            if (T.C < 2 || T.n_coeffs < 1 || T.n_coeffs > 16) return fail(c, ALEA_ERR_INVALID, "bad Drummond term");
            D.C = T.C;
            D.gamma = T.gamma;
            D.L = T.L;
            D.ncoef = T.n_coeffs;
            for (int k = 0; k < T.n_coeffs; ++k) D.dc[k] = T.dcoeffs[k];
            double ipw = 1.0;
            for (int i = 0; i < T.C; ++i) ipw *= -T.L;
            D.alpha1 = T.gamma / ipw + D.dc[0] * static_cast<double>(T.C) / T.L;
        } else {
            return fail(c, ALEA_ERR_UNSUPPORTED, "three-dimensional pair terms are Padé or Drummond");
        }
    }
    c->h_opt.clear();
    s.pair_by_group = 0;
    s.nkJ = 0;
    s.o_rho = static_cast<int>(o);
    s.hot = static_cast<int>(round4(o));
    s.rec = s.hot;
    std::vector<std::vector<double>> poly_tables;
    std::vector<double> ek3;
    s.ewald = in->ewald.enabled;
    if (s.ewald) {
        const alea_gpu_ewald& E = in->ewald;
        const alea_gpu_kset& K = E.kset;
        if (!s.periodic) return fail(c, ALEA_ERR_INVALID, "Ewald in an open cell");
        if (!E.long_range.scaled || E.long_range.n_knots < 2 || K.n_k < 0 ||
            (K.n_k > 0 && (!K.kx || !K.ky || !K.kz || !K.weight)))
            return fail(c, ALEA_ERR_INVALID, "bad 3-D Ewald tables (the k set needs kz)");
        s.esp.r_cut = E.long_range.r_cut;
        s.esp.inv_delta = E.long_range.inv_delta;
        s.esp.n_knots = E.long_range.n_knots;
        put(E.long_range.scaled, 3 * E.long_range.n_knots * 8, reinterpret_cast<const void**>(&s.esp.scaled));
        poly_tables.push_back(hermite_to_monomial(E.long_range.scaled, E.long_range.n_knots));
        put(poly_tables.back().data(), poly_tables.back().size() * 8, reinterpret_cast<const void**>(&s.esp.poly));
        s.e_rcut = E.r_cut;
        s.e_inv_eps = E.inv_eps;
        s.e_const = E.constant;
        s.enk = K.n_k;
        for (int k = 0; k < K.n_k; ++k) {
            ek3.push_back(K.kx[k]);
            ek3.push_back(K.ky[k]);
            ek3.push_back(K.kz[k]);
        }
        if (s.enk > 0) {
            put(ek3.data(), ek3.size() * 8, reinterpret_cast<const void**>(&s.ek3));
            put(K.weight, 8 * s.enk, reinterpret_cast<const void**>(&s.ew));
        }
    }
    if (in->n_coulomb < 0 || in->n_coulomb > kMaxCoulomb) return fail(c, ALEA_ERR_INVALID, "bad n_coulomb");
    s.ncoul = in->n_coulomb;
    for (int k = 0; k < s.ncoul; ++k) {
        const alea_gpu_coulomb& C = in->coulomb[k];
        s.coul[k][0] = C.a_first;
        s.coul[k][1] = C.a_last;
        s.coul[k][2] = C.b_first;
        s.coul[k][3] = C.b_last;
        s.coul_coef[k] = C.coef;
    }
    if (in->n_inverse_power != 0)
        return fail(c, ALEA_ERR_UNSUPPORTED, "three-dimensional systems take no inverse-power terms");
    s.nip = 0;
    s.ip_tail = 0.0;
    const Ziggurat z = make_ziggurat();
    put(z.k, sizeof z.k, reinterpret_cast<const void**>(&s.zk));
    put(z.w, sizeof z.w, reinterpret_cast<const void**>(&s.zw));
    put(z.f, sizeof z.f, reinterpret_cast<const void**>(&s.zf));
    s.zr = z.r;
    // shared memory after the hot part (alea_bf3d.cu's view3)
    long m = s.hot;
    auto take = [&](long n) {
        const long at = m;
        m += round4(std::max(n, 1L));
        return static_cast<int>(at);
    };
    s.t_newpos = take(4);
    s.t_misc = take(32);
    s.t_red = take(96);
    s.t_col = take(s.maxN);
    s.t_work = static_cast<int>(m);
    for (int d = 0; d < s.nbf; ++d) {
        DevBF& D = s.bf[d];
        D.pX = take(3 * D.n);
        D.pA = take(D.n * D.n);
        D.pF = take(3 * D.n);
        D.pM = take(8);
    }
    s.t_mwork = static_cast<int>(m);
    const long N = s.maxN;
    // the moves' layout ends with each determinant's Gauss-Jordan multipliers and
    // row exchanges (2N); the refresh's work area (from t_work): M, orbital rows,
    // G, T, slice sums (48N for the per-particle warps when N < 12)
    s.t_mtotal = static_cast<int>(s.t_mwork + s.nbf * round4(2 * N));
    const long refresh = 8 * N * N + 18 * N + (N < 12 ? 36 * N : 0);
    const long total = std::max(static_cast<long>(s.t_mtotal), s.t_work + round4(refresh));
    s.t_total = static_cast<int>(total);
    s.f_total = 0;
    c->smem = static_cast<size_t>(total) * 8;
    if (c->smem > 227 * 1024)
        return fail(c, ALEA_ERR_UNSUPPORTED,
                    "walker state needs " + std::to_string(c->smem) + " bytes of shared memory (> 227 KB)");
    {
        uint64_t h = 1469598103934665603ULL;
        auto mix = [&h](const void* p, size_t n) {
            const unsigned char* b = static_cast<const unsigned char*>(p);
            for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ULL;
        };
        mix(&s, sizeof s);
        mix(ar.bytes.data(), ar.bytes.size());
        c->fingerprint = h;
    }
    CUDA_TRY(c, cudaMallocAsync(&c->arena, std::max<size_t>(ar.bytes.size(), 256), c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->arena, ar.bytes.data(), ar.bytes.size(), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (const Patch& p : patches) *p.slot = static_cast<char*>(c->arena) + p.off;
    c->orbital_opts = 0;
    return ALEA_OK;
}

int ensure_streams(alea_gpu_ctx* c, int n) {
    if (n > c->streams_cap) {
        if (c->streams) cudaFreeAsync(c->streams, c->stream);
        c->streams = nullptr;
        CUDA_TRY(c, cudaMallocAsync(&c->streams, sizeof(uint64_t) * 4 * static_cast<size_t>(n), c->stream));
        c->streams_cap = n;
    }
    return ALEA_OK;
}

int ensure_randoms(alea_gpu_ctx* c, int sweeps) {
    if (sweeps > c->rnd_sweeps) {
        if (c->randoms) cudaFreeAsync(c->randoms, c->stream);
        c->randoms = nullptr;
        const size_t n = static_cast<size_t>(sweeps) * c->sys.np * (c->sys.dim + 1) * c->capacity;
        CUDA_TRY(c, cudaMallocAsync(&c->randoms, n * 8, c->stream));
        c->rnd_sweeps = sweeps;
    }
    return ALEA_OK;
}

int set_sigma(alea_gpu_ctx* c, double tau) {
    if (tau == c->sigma_tau) return ALEA_OK;
    std::vector<double> sg(c->h_inv_mass.size());
    for (size_t i = 0; i < sg.size(); ++i) sg[i] = std::sqrt(tau * c->h_inv_mass[i]);
    CUDA_TRY(c, copy_in(c, c->d_sigma, sg.data(), sg.size() * 8));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->sigma_tau = tau;
    return ALEA_OK;
}

double* records(alea_gpu_ctx* c) { return c->rec[c->cur]; }

int read_scalars(alea_gpu_ctx* c, int slot, std::vector<double>& out) {
    out.resize(c->nw);
    if (c->nw == 0) return ALEA_OK;
    ++c->launches;
    scalar_kernel<<<(c->nw + 255) / 256, 256, 0, c->stream>>>(records(c), c->nw, c->sys.rec,
                                                              c->sys.o_scal + slot, c->d_buf);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, copy_out(c, out.data(), c->d_buf, 8 * c->nw));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

// Several scalar slots of every walker in one transfer: plane k of `slots`
// lands in out[k] (one copy and one synchronisation for all of them).
int read_pack(alea_gpu_ctx* c, std::initializer_list<int> slots, std::initializer_list<std::vector<double>*> out) {
    const int nw = c->nw;
    int k = 0;
    for (int slot : slots) {
        ++c->launches;
        scalar_kernel<<<(nw + 255) / 256, 256, 0, c->stream>>>(records(c), nw, c->sys.rec, c->sys.o_scal + slot,
                                                                c->d_buf + static_cast<size_t>(k) * nw);
        CUDA_TRY(c, cudaGetLastError());
        ++k;
    }
    CUDA_TRY(c, copy_out(c, c->h_stage, c->d_buf, 8L * k * nw));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    k = 0;
    for (std::vector<double>* v : out) {
        v->assign(c->h_stage + static_cast<long>(k) * nw, c->h_stage + static_cast<long>(k + 1) * nw);
        ++k;
    }
    return ALEA_OK;
}

int check_errors(alea_gpu_ctx* c) {
    std::vector<double> e;
    if (int rc = read_scalars(c, S_ERR, e)) return rc;
    for (int w = 0; w < c->nw; ++w)
        if (e[w] != 0.0)
            return fail(c, ALEA_ERR_SINGULAR,
                        "walker " + std::to_string(w) + ": accepted determinant is singular or nonfinite");
    return ALEA_OK;
}

int launch_evaluate(alea_gpu_ctx* c) {
    if (c->nw == 0) return ALEA_OK;
    ++c->launches;
    if (c->sys.dim == 3)
        CUDA_TRY(c, launch_evaluate3(c->nw, c->smem, c->stream, c->sys, records(c)));
    else
        CUDA_TRY(c, launch_evaluate(c->nt, c->nw, c->smem, c->stream, c->sys, records(c), c->pairs, c->npair));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return check_errors(c);
}

// One sweep-kernel launch (VMC step or DMC advance) with its randoms.
int run_sweep(alea_gpu_ctx* c, int mode, int n_sub, double tau, int drift, double etrial, double eref,
              double e_cut, double e_max, bool check = true) {
    if (c->nw == 0) return ALEA_OK;
    if (c->n_streams < 1) return fail(c, ALEA_ERR_INVALID, "no random streams (alea_gpu_set_streams)");
    if (n_sub < 1) return fail(c, ALEA_ERR_INVALID, "n_substeps must be >= 1");
    if (int rc = ensure_randoms(c, n_sub)) return rc;
    if (int rc = set_sigma(c, tau)) return rc;
    const long stride = c->nw;
    const int nt = std::min(c->n_streams, c->nw);
    ++c->launches;
    draw_kernel<<<(nt + 127) / 128, 128, 0, c->stream>>>(c->streams, c->n_streams, c->nw, c->sys.np, stride,
                                                         n_sub, c->sys.zk, c->sys.zw, c->sys.zf, c->sys.zr,
                                                         c->randoms, c->sys.dim);
    CUDA_TRY(c, cudaGetLastError());
    SweepParams prm{};
    prm.mode = mode;
    prm.n_sub = n_sub;
    prm.drift = drift;
    prm.tau = tau;
    prm.sigma = c->d_sigma;
    prm.etrial = etrial;
    prm.eref = eref;
    prm.e_cut = e_cut;
    prm.e_max = e_max;
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    ++c->launches;
    if (c->sys.dim == 3)
        CUDA_TRY(c, launch_sweep3(c->nw, c->smem, c->stream, c->sys, records(c), c->randoms, stride, prm));
    else
        CUDA_TRY(c, launch_sweep(c->nt, c->nw, c->smem, c->stream, c->sys, records(c), c->randoms, stride, prm,
                                 c->pairs, c->npair));
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    return check ? check_errors(c) : ALEA_OK;
}

// ───────────────────────── allocation-free VMC step ─────────────────────
//
// Scratch of alea_gpu_vmc_step_noalloc: the sweep's random numbers
// [(sweep·np + p)·3·nw + d·nw + w], then the step's reduced statistics.  A
// file-scope device array exists once per device, so every context on a
// device shares it; each call writes all of the scratch it reads (randoms by
// draw_kernel, statistics by noalloc_stats_kernel) before reading it, so
// nothing in it needs to start at zero.
constexpr size_t kNoAllocRandoms = size_t(1) << 20;   // doubles (8 MiB)
constexpr size_t kNoAllocStats = 32;                  // doubles, 4 used
static_assert(kNoAllocRandoms == ALEA_GPU_NOALLOC_RANDOMS, "header and scratch size disagree");
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocRandoms + kNoAllocStats];

// One block of 256 threads: Σ E_L, Σ E_L², Σ accepted moves and max |error
// flag| over the walkers, written (not accumulated) to out[0..3].
__global__ void __launch_bounds__(256) noalloc_stats_kernel(const double* records, int nw, long rec,
                                                             int o_scal, double* out) {
    __shared__ double red[4][256];
    double e = 0.0, e2 = 0.0, na = 0.0, er = 0.0;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        const double* r = records + static_cast<size_t>(w) * rec + o_scal;
        const double el = r[S_EL];
        e += el;
        e2 += el * el;
        na += r[S_NACC];
        er = fmax(er, fabs(r[S_ERR]));
    }
    red[0][threadIdx.x] = e;
    red[1][threadIdx.x] = e2;
    red[2][threadIdx.x] = na;
    red[3][threadIdx.x] = er;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] += red[1][threadIdx.x + h];
            red[2][threadIdx.x] += red[2][threadIdx.x + h];
            red[3][threadIdx.x] = fmax(red[3][threadIdx.x], red[3][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

// sqrt(τ/m) per coordinate from the device's inverse-mass table (the host's
// IEEE product and square root, so equal to what alea_gpu_vmc_step stages).
__global__ void sigma_kernel(double* sigma, const double* inv_mass, int n, double tau) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) sigma[i] = sqrt(tau * inv_mass[i]);
}

}  // namespace

// ───────────────────────── C ABI ────────────────────────────────────────

extern "C" {

int alea_gpu_abi_version(void) { return ALEA_GPU_ABI_VERSION; }

const char* alea_gpu_last_error(const alea_gpu_ctx* ctx) {
    return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int alea_gpu_create(const alea_gpu_system* sys, int device, int capacity, alea_gpu_ctx** out) {
    if (!out) return fail(nullptr, ALEA_ERR_INVALID, "null output pointer");
    *out = nullptr;
    if (capacity < 1) return fail(nullptr, ALEA_ERR_INVALID, "capacity must be >= 1");
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0)
        return fail(nullptr, ALEA_ERR_CUDA, "no CUDA device");
    if (device < 0 || device >= n_dev) return fail(nullptr, ALEA_ERR_INVALID, "bad device index");
    auto* c = new alea_gpu_ctx();
    c->device = device;
    c->capacity = capacity;
    auto bail = [&](int rc) {
        g_create_error = c->err;
        alea_gpu_destroy(c);
        return rc;
    };
    if (cudaSetDevice(device) != cudaSuccess) {
        c->err = "cudaSetDevice failed";
        return bail(ALEA_ERR_CUDA);
    }
    // Device memory is stream-ordered (cudaMallocAsync on the context's own
    // stream, from the device's pool kept warm), so creating or destroying a
    // context never waits for other contexts' work on the device.
    keep_pool_warm(device);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        c->err = "cudaStreamCreate failed";
        return bail(ALEA_ERR_CUDA);
    }
    if (int rc = build_system(c, sys)) return bail(rc);
    const DevSys& s = c->sys;
    const size_t recb = static_cast<size_t>(s.rec) * 8 * capacity;
    cudaStream_t st = c->stream;
    if (cudaMallocAsync(&c->rec[0], recb, st) != cudaSuccess || cudaMallocAsync(&c->rec[1], recb, st) != cudaSuccess ||
        cudaMallocAsync(&c->d_buf, static_cast<size_t>(std::max(s.np * s.dim, 8)) * 8 * capacity, st) != cudaSuccess ||
        cudaMallocAsync(&c->d_sigma, static_cast<size_t>(s.np) * s.dim * 8, st) != cudaSuccess ||
        cudaMallocAsync(&c->d_src, sizeof(int) * static_cast<size_t>(capacity), st) != cudaSuccess ||
        cudaMallocAsync(&c->d_mask, static_cast<size_t>(capacity), st) != cudaSuccess ||
        (c->h_stage = static_cast<double*>(pinned_acquire(64 * static_cast<size_t>(capacity)))) == nullptr ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess) {
        c->err = "device allocation failed";
        return bail(ALEA_ERR_NOMEM);
    }
    cudaMemsetAsync(c->rec[0], 0, recb, st);
    cudaMemsetAsync(c->rec[1], 0, recb, st);
    // pair list i < j for the Ewald real-space sum
    std::vector<int2> pl;
    for (int i = 0; i < s.np; ++i)
        for (int j = i + 1; j < s.np; ++j) pl.push_back(make_int2(i, j));
    c->npair = static_cast<int>(pl.size());
    if (c->npair > 0) {
        if (cudaMallocAsync(&c->pairs, pl.size() * sizeof(int2), st) != cudaSuccess ||
            cudaMemcpyAsync(c->pairs, pl.data(), pl.size() * sizeof(int2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            c->err = "device allocation failed";
            return bail(ALEA_ERR_NOMEM);
        }
    }
    c->nt = pick_threads(s);
    // the one-warp layouts (f_total) are launched at their own size
    const size_t reserve = std::max(c->smem, static_cast<size_t>(s.f_total) * 8);
    if (reserve_smem(reserve) != cudaSuccess) {
        c->err = "cannot reserve " + std::to_string(reserve) + " bytes of shared memory";
        return bail(ALEA_ERR_UNSUPPORTED);
    }
    *out = c;
    return ALEA_OK;
}

namespace {
void fw_free(alea_gpu_ctx* c);
}  // namespace

int alea_gpu_destroy(alea_gpu_ctx* c) {
    if (!c) return ALEA_OK;
    for (void* p : {static_cast<void*>(c->arena), static_cast<void*>(c->rec[0]), static_cast<void*>(c->rec[1]),
                    static_cast<void*>(c->randoms), static_cast<void*>(c->streams), static_cast<void*>(c->pairs),
                    static_cast<void*>(c->d_buf), static_cast<void*>(c->d_sigma), static_cast<void*>(c->d_src),
                    static_cast<void*>(c->d_mask), static_cast<void*>(c->d_opt), static_cast<void*>(c->d_opt_out),
                    static_cast<void*>(c->d_opt_grad), static_cast<void*>(c->d_opt_scratch),
                    static_cast<void*>(c->d_sys)})
        if (p && c->stream) cudaFreeAsync(p, c->stream);
    if (c->stream) alea_gpu::est_free(c->est, c->stream);
    if (c->stream) fw_free(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    pinned_release(c->h_stage, 64 * static_cast<size_t>(c->capacity));
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ALEA_OK;
}

int alea_gpu_num_walkers(const alea_gpu_ctx* c, int* nw) {
    if (!c || !nw) return ALEA_ERR_INVALID;
    *nw = c->nw;
    return ALEA_OK;
}

int alea_gpu_upload_walkers(alea_gpu_ctx* c, const double* positions, int nw) {
    const Phase phase("alea.upload");
    if (!c) return ALEA_ERR_INVALID;
    if (nw < 1 || nw > c->capacity) return fail(c, ALEA_ERR_NOMEM, "walker count exceeds the capacity");
    if (!positions) return fail(c, ALEA_ERR_INVALID, "null positions");
    for (long i = 0, n = static_cast<long>(c->sys.np) * c->sys.dim * nw; i < n; ++i)
        if (!std::isfinite(positions[i]))
            return fail(c, ALEA_ERR_INVALID, "walker positions must be finite (entry " + std::to_string(i) + ")");
    cudaSetDevice(c->device);
    c->cur = 0;
    c->nw = nw;
    const DevSys& s = c->sys;
    CUDA_TRY(c, cudaMemsetAsync(records(c), 0, static_cast<size_t>(s.rec) * 8 * nw, c->stream));
    CUDA_TRY(c, copy_in(c, c->d_buf, positions, static_cast<size_t>(s.np) * s.dim * nw * 8));
    const long n = static_cast<long>(s.np) * s.dim * nw;
    ++c->launches;
    from_soa_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, c->stream>>>(records(c), nw, s.rec, s.o_pos,
                                                                             s.np * s.dim, c->d_buf);
    ++c->launches;
    set_scalar_kernel<<<(nw + 255) / 256, 256, 0, c->stream>>>(records(c), nw, s.rec, s.o_scal + S_WEIGHT, 1.0);
    CUDA_TRY(c, cudaGetLastError());
    c->next_id = 1.0;
    return launch_evaluate(c);
}

int alea_gpu_evaluate(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    return launch_evaluate(c);
}

int alea_gpu_download_phase(alea_gpu_ctx* c, double* phase_gradients, double* phase_laplacians,
                            double* local_energy_imag) {
    if (!c) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    const DevSys& s = c->sys;
    if (!s.cplx) return fail(c, ALEA_ERR_INVALID, "the trial function is real: it has no phase planes");
    const int nw = c->nw;
    if (nw == 0) return ALEA_OK;
    const long n = static_cast<long>(s.np) * 2 * nw;
    const int grid = static_cast<int>((n + 255) / 256);
    for (int which = 0; which < 2; ++which) {
        double* dst = which == 0 ? phase_gradients : phase_laplacians;
        if (!dst) continue;
        ++c->launches;
        to_soa_kernel<<<grid, 256, 0, c->stream>>>(records(c), nw, s.rec, which == 0 ? s.o_pg : s.o_pl,
                                                   s.np * 2, c->d_buf);
        CUDA_TRY(c, cudaGetLastError());
        CUDA_TRY(c, copy_out(c, dst, c->d_buf, n * 8));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    }
    if (local_energy_imag) {
        std::vector<double> tmp;
        if (int rc = read_scalars(c, S_ELI, tmp)) return rc;
        std::copy(tmp.begin(), tmp.end(), local_energy_imag);
    }
    return ALEA_OK;
}

int alea_gpu_download_walkers(alea_gpu_ctx* c, double* positions, double* log_psi, double* gradients,
                              double* laplacians, double* local_energy, double* weights) {
    if (!c) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    const DevSys& s = c->sys;
    const int nw = c->nw;
    if (nw == 0) return ALEA_OK;
    const long n = static_cast<long>(s.np) * s.dim * nw;
    const int grid = static_cast<int>((n + 255) / 256);
    auto plane = [&](int off, double* dst) -> int {
        ++c->launches;
        to_soa_kernel<<<grid, 256, 0, c->stream>>>(records(c), nw, s.rec, off, s.np * s.dim, c->d_buf);
        CUDA_TRY(c, cudaGetLastError());
        CUDA_TRY(c, copy_out(c, dst, c->d_buf, n * 8));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        return ALEA_OK;
    };
    if (positions)
        if (int rc = plane(s.o_pos, positions)) return rc;
    if (gradients || laplacians) {
        std::vector<double> a(n), b(n);
        for (int which = 0; which < 2; ++which) {
            double* dst = which == 0 ? gradients : laplacians;
            if (!dst) continue;
            if (int rc = plane(which == 0 ? s.o_sg : s.o_sl, a.data())) return rc;
            if (int rc = plane(which == 0 ? s.o_jg : s.o_jl, b.data())) return rc;
            for (long i = 0; i < n; ++i) dst[i] = a[i] + b[i];
            if (int rc = plane(which == 0 ? s.o_kg : s.o_kl, b.data())) return rc;
            for (long i = 0; i < n; ++i) dst[i] += b[i];
        }
    }
    std::vector<double> tmp;
    if (log_psi) {
        if (int rc = read_scalars(c, S_LOGPSI, tmp)) return rc;
        std::copy(tmp.begin(), tmp.end(), log_psi);
    }
    if (local_energy) {
        if (int rc = read_scalars(c, S_EL, tmp)) return rc;
        std::copy(tmp.begin(), tmp.end(), local_energy);
    }
    if (weights) {
        if (int rc = read_scalars(c, S_WEIGHT, tmp)) return rc;
        std::copy(tmp.begin(), tmp.end(), weights);
    }
    return ALEA_OK;
}

int alea_gpu_move(alea_gpu_ctx* c, int p, const double* new_pos, const uint8_t* accept, double* log_ratio,
                  double* phase, double* new_grad, double* new_lap) {
    if (!c || !new_pos) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_move: two-dimensional systems only");
    if (c->sys.f32)
        return fail(c, ALEA_ERR_UNSUPPORTED, "single moves run in FP64: set the precision back to FP64 first");
    const DevSys& s = c->sys;
    if (p < 0 || p >= s.np) return fail(c, ALEA_ERR_INVALID, "particle index out of range");
    cudaSetDevice(c->device);
    const int nw = c->nw;
    if (nw == 0) return ALEA_OK;
    double* d_np = c->d_buf;
    double* d_out = c->d_buf + 2 * nw;
    if (static_cast<long>(8) * nw > static_cast<long>(std::max(s.np * 2, 8)) * c->capacity)
        return fail(c, ALEA_ERR_NOMEM, "staging buffer too small");
    CUDA_TRY(c, copy_in(c, d_np, new_pos, 16L * nw));
    if (accept) CUDA_TRY(c, copy_in(c, c->d_mask, accept, nw));
    ++c->launches;
    CUDA_TRY(c, launch_move(c->nt, nw, c->smem, c->stream, s, records(c), p, d_np,
                            accept ? c->d_mask : nullptr, d_out));
    std::vector<double> out(6L * nw);
    CUDA_TRY(c, copy_out(c, out.data(), d_out, 48L * nw));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    for (int w = 0; w < nw; ++w) {
        if (log_ratio) log_ratio[w] = out[w];
        if (phase) phase[w] = out[nw + w];
        if (new_grad) {
            new_grad[w] = out[2 * nw + w];
            new_grad[nw + w] = out[3 * nw + w];
        }
        if (new_lap) {
            new_lap[w] = out[4 * nw + w];
            new_lap[nw + w] = out[5 * nw + w];
        }
    }
    return accept ? check_errors(c) : ALEA_OK;
}

int alea_gpu_set_precision(alea_gpu_ctx* c, int precision) {
    if (!c) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2 && precision == ALEA_PRECISION_FP32)
        return fail(c, ALEA_ERR_UNSUPPORTED, "the FP32 form runs two-dimensional systems only");
    cudaSetDevice(c->device);
    if (precision == ALEA_PRECISION_FP32) {
        if (c->nt != 32 || !f32_sweep_eligible(c->sys))
            return fail(c, ALEA_ERR_UNSUPPORTED,
                        "the FP32 form takes real determinants and Pade/Drummond pair terms of at most 64 particles");
        c->sys.f32 = 1;
        return ALEA_OK;
    }
    if (precision != ALEA_PRECISION_FP64) return fail(c, ALEA_ERR_INVALID, "precision must be FP64 or FP32");
    if (!c->sys.f32) return ALEA_OK;
    c->sys.f32 = 0;
    return c->nw > 0 ? launch_evaluate(c) : ALEA_OK;   // FP64 inverses and orbital rows again
}

// The reference's split of a move (ParticleBatch::propose_move_batch,
// WavefunctionComponent::ratio_batch, commit), each step alea_gpu_move's
// arithmetic: the proposal is kept on the host until committed.
int alea_gpu_propose(alea_gpu_ctx* c, int p, const double* new_pos) {
    if (!c || !new_pos) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_propose: two-dimensional systems only");
    if (p < 0 || p >= c->sys.np) return fail(c, ALEA_ERR_INVALID, "particle index out of range");
    c->prop_p = p;
    c->prop_pos.assign(new_pos, new_pos + 2L * c->nw);
    return ALEA_OK;
}

int alea_gpu_ratio(alea_gpu_ctx* c, int p, double* log_ratio, double* phase, double* new_grad, double* new_lap) {
    if (!c) return ALEA_ERR_INVALID;
    if (p != c->prop_p || c->prop_pos.size() != 2u * c->nw)
        return fail(c, ALEA_ERR_INVALID, "ratio: no proposal of this particle (alea_gpu_propose)");
    return alea_gpu_move(c, p, c->prop_pos.data(), nullptr, log_ratio, phase, new_grad, new_lap);
}

int alea_gpu_commit(alea_gpu_ctx* c, int p, const uint8_t* mask) {
    if (!c || !mask) return ALEA_ERR_INVALID;
    if (p != c->prop_p || c->prop_pos.size() != 2u * c->nw)
        return fail(c, ALEA_ERR_INVALID, "commit: no proposal of this particle (alea_gpu_propose)");
    const int rc = alea_gpu_move(c, p, c->prop_pos.data(), mask, nullptr, nullptr, nullptr, nullptr);
    c->prop_p = -1;
    c->prop_pos.clear();
    return rc;
}

int alea_gpu_local_energy(alea_gpu_ctx* c, double* el) {
    if (!c || !el) return ALEA_ERR_INVALID;
    if (int rc = alea_gpu_measure(c)) return rc;
    std::vector<double> v;
    if (int rc = read_scalars(c, S_EL, v)) return rc;
    std::copy(v.begin(), v.end(), el);
    return ALEA_OK;
}

int alea_gpu_measure(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->nw == 0) return ALEA_OK;
    // the FP32 form keeps no orbital rows to refresh from; a 3-D walker is evaluated anew
    if (c->sys.f32 || c->sys.dim == 3) return launch_evaluate(c);
    ++c->launches;
    CUDA_TRY(c, launch_measure(c->nt, c->nw, c->smem, c->stream, c->sys, records(c), c->pairs, c->npair));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

int alea_gpu_set_rng_streams(alea_gpu_ctx* c, uint64_t stage_seed, uint64_t stream_kind, int n_streams) {
    return alea_gpu_set_streams(c, stage_seed, stream_kind, n_streams);
}

int alea_gpu_vmc_steps(alea_gpu_ctx* c, const alea_gpu_vmc_params* prm, int n_steps, alea_gpu_step_stats* out) {
    if (!c || !prm || n_steps < 0) return ALEA_ERR_INVALID;
    alea_gpu_step_stats tot{};
    for (int i = 0; i < n_steps; ++i) {
        alea_gpu_step_stats st{};
        if (int rc = alea_gpu_vmc_step(c, prm, &st)) return rc;
        tot.energy_sum += st.energy_sum;
        tot.energy_sq_sum += st.energy_sq_sum;
        tot.weight_sum += st.weight_sum;
        tot.n_accepted += st.n_accepted;
        tot.n_proposed += st.n_proposed;
        tot.n_walkers = st.n_walkers;
    }
    if (out) *out = tot;
    return ALEA_OK;
}

int alea_gpu_dmc_steps(alea_gpu_ctx* c, const alea_gpu_dmc_params* prm, int n_steps, uint64_t* branch_state,
                       int target, alea_gpu_step_stats* out) {
    if (!c || !prm || !branch_state || n_steps < 0) return ALEA_ERR_INVALID;
    alea_gpu_step_stats tot{};
    for (int i = 0; i < n_steps; ++i) {
        alea_gpu_step_stats st{};
        if (int rc = alea_gpu_dmc_advance(c, prm, &st)) return rc;
        if (int rc = alea_gpu_dmc_branch(c, branch_state, target)) return rc;
        tot.energy_sum += st.energy_sum;
        tot.energy_sq_sum += st.energy_sq_sum;
        tot.weight_sum += st.weight_sum;
        tot.n_accepted += st.n_accepted;
        tot.n_proposed += st.n_proposed;
        tot.n_cut += st.n_cut;
        tot.n_walkers = c->nw;
    }
    if (out) *out = tot;
    return ALEA_OK;
}

int alea_gpu_set_streams(alea_gpu_ctx* c, uint64_t seed, uint64_t kind, int n) {
    if (!c || n < 1) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    if (int rc = ensure_streams(c, n)) return rc;
    std::vector<uint64_t> st(4L * n);
    for (int t = 0; t < n; ++t) {
        HostXo x(stream_seed(seed, kind, static_cast<uint64_t>(t)));
        for (int k = 0; k < 4; ++k) st[4L * t + k] = x.s[k];
    }
    CUDA_TRY(c, copy_in(c, c->streams, st.data(), st.size() * 8));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->n_streams = n;
    return ALEA_OK;
}

int alea_gpu_vmc_step(alea_gpu_ctx* c, const alea_gpu_vmc_params* prm, alea_gpu_step_stats* out) {
    const Phase phase("alea.vmc_step");
    if (!c || !prm) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    if (int rc = run_sweep(c, 0, prm->n_substeps, prm->tau, prm->use_drift, 0, 0, 0, 0)) return rc;
    if (out) {
        std::vector<double> el, na;
        if (int rc = read_scalars(c, S_EL, el)) return rc;
        if (int rc = read_scalars(c, S_NACC, na)) return rc;
        *out = alea_gpu_step_stats{};
        for (int w = 0; w < c->nw; ++w) {
            out->energy_sum += el[w];
            out->energy_sq_sum += el[w] * el[w];
            out->n_accepted += static_cast<int64_t>(na[w]);
        }
        out->weight_sum = c->nw;
        out->n_proposed = static_cast<int64_t>(prm->n_substeps) * c->sys.np * c->nw;
        out->n_walkers = c->nw;
    }
    return ALEA_OK;
}

int alea_gpu_vmc_step_noalloc(alea_gpu_ctx* c, const alea_gpu_vmc_params* prm, alea_gpu_step_stats* out) {
    if (!c || !prm) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    if (c->nw == 0) {
        if (out) *out = alea_gpu_step_stats{};
        return ALEA_OK;
    }
    if (c->n_streams < 1) return fail(c, ALEA_ERR_INVALID, "no random streams (alea_gpu_set_streams)");
    if (prm->n_substeps < 1) return fail(c, ALEA_ERR_INVALID, "n_substeps must be >= 1");
    if (c->sys.dim != 2)
        return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_vmc_step_noalloc: two-dimensional systems only");
    const size_t need = static_cast<size_t>(prm->n_substeps) * c->sys.np * 3 * c->nw;
    if (need > kNoAllocRandoms)
        return fail(c, ALEA_ERR_INVALID,
                    "alea_gpu_vmc_step_noalloc: n_substeps x particles x 3 x walkers = " + std::to_string(need) +
                        " random numbers exceed the static scratch of " + std::to_string(kNoAllocRandoms));
    if (!c->noalloc_scratch) {   // set-up, once per context (and so per device)
        void* p = nullptr;
        CUDA_TRY(c, cudaGetSymbolAddress(&p, g_noalloc_scratch));
        c->noalloc_scratch = static_cast<double*>(p);
    }
    if (prm->tau != c->sigma_tau) {   // sqrt(τ/m) per coordinate, computed on the device
        const int n = static_cast<int>(c->h_inv_mass.size());
        ++c->launches;
        sigma_kernel<<<(n + 127) / 128, 128, 0, c->stream>>>(c->d_sigma, c->sys.inv_mass, n, prm->tau);
        CUDA_TRY(c, cudaGetLastError());
        c->sigma_tau = prm->tau;
    }
    double* rnd = c->noalloc_scratch;
    double* stats = c->noalloc_scratch + kNoAllocRandoms;
    const long stride = c->nw;
    const int nt = std::min(c->n_streams, c->nw);
    ++c->launches;
    draw_kernel<<<(nt + 127) / 128, 128, 0, c->stream>>>(c->streams, c->n_streams, c->nw, c->sys.np, stride,
                                                         prm->n_substeps, c->sys.zk, c->sys.zw, c->sys.zf,
                                                         c->sys.zr, rnd, c->sys.dim);
    CUDA_TRY(c, cudaGetLastError());
    SweepParams sp{};
    sp.mode = 0;
    sp.n_sub = prm->n_substeps;
    sp.drift = prm->use_drift;
    sp.tau = prm->tau;
    sp.sigma = c->d_sigma;
    ++c->launches;
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    CUDA_TRY(c, launch_sweep(c->nt, c->nw, c->smem, c->stream, c->sys, records(c), rnd, stride, sp, c->pairs,
                             c->npair));
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    ++c->launches;
    noalloc_stats_kernel<<<1, 256, 0, c->stream>>>(records(c), c->nw, c->sys.rec, c->sys.o_scal, stats);
    CUDA_TRY(c, cudaGetLastError());
    double h[4];
    CUDA_TRY(c, copy_out(c, h, stats, sizeof h));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    if (h[3] != 0.0) return fail(c, ALEA_ERR_SINGULAR, "a walker's accepted determinant is singular or nonfinite");
    if (out) {
        *out = alea_gpu_step_stats{};
        out->energy_sum = h[0];
        out->energy_sq_sum = h[1];
        out->n_accepted = static_cast<int64_t>(h[2]);
        out->weight_sum = c->nw;
        out->n_proposed = static_cast<int64_t>(prm->n_substeps) * c->sys.np * c->nw;
        out->n_walkers = c->nw;
    }
    return ALEA_OK;
}

int alea_gpu_dmc_advance(alea_gpu_ctx* c, const alea_gpu_dmc_params* prm, alea_gpu_step_stats* out) {
    const Phase phase("alea.dmc_advance");
    if (!c || !prm) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    if (int rc = run_sweep(c, 1, prm->n_substeps, prm->tau, 1, prm->e_trial, prm->e_ref, prm->e_cut, prm->e_max,
                           false))
        return rc;
    // weights, energies, counters and error flags in one transfer
    std::vector<double> err;
    if (int rc = read_pack(c, {S_WEIGHT, S_EL, S_NACC, S_NCUT, S_ERR}, {&c->h_w, &c->h_el, &c->h_nacc, &c->h_ncut, &err}))
        return rc;
    for (int w = 0; w < c->nw; ++w)
        if (err[w] != 0.0)
            return fail(c, ALEA_ERR_SINGULAR,
                        "walker " + std::to_string(w) + ": accepted determinant is singular or nonfinite");
    if (out) {
        *out = alea_gpu_step_stats{};
        // Σ w E and Σ w per crowd, then over crowds (dmc.cpp:713-724)
        const int nw = c->nw;
        const int nact = std::min(c->n_streams, nw);
        const int base = nw / nact, rem = nw % nact;
        for (int t = 0; t < nact; ++t) {
            const int w0 = t * base + std::min(t, rem), cnt = base + (t < rem ? 1 : 0);
            double e = 0.0, ws = 0.0;
            for (int w = w0; w < w0 + cnt; ++w) {
                e += c->h_w[w] * c->h_el[w];
                ws += c->h_w[w];
            }
            out->energy_sum += e;
            out->weight_sum += ws;
        }
        for (int w = 0; w < nw; ++w) {
            out->n_accepted += static_cast<int64_t>(c->h_nacc[w]);
            out->n_cut += static_cast<int64_t>(c->h_ncut[w]);
            out->energy_sq_sum += c->h_w[w] * c->h_el[w] * c->h_el[w];
        }
        out->n_proposed = static_cast<int64_t>(prm->n_substeps) * c->sys.np * nw;
        out->n_walkers = nw;
    }
    return ALEA_OK;
}

int alea_gpu_dmc_branch(alea_gpu_ctx* c, uint64_t* state, int target) {
    const Phase phase("alea.dmc_branch");
    if (!c || !state || target < 1) return ALEA_ERR_INVALID;
    cudaSetDevice(c->device);
    const int n = c->nw;
    if (n == 0) return ALEA_OK;
    std::vector<double> w, ids, par;
    if (int rc = read_pack(c, {S_WEIGHT, S_ID, S_PARENT}, {&w, &ids, &par})) return rc;
    HostXo rng;
    std::memcpy(rng.s, state, 32);
    std::vector<int> src;
    src.reserve(2 * target + 2);
    const size_t n_max = 2 * static_cast<size_t>(target) + 1, n_min = static_cast<size_t>(target) / 5 + 1;
    // Multiplicities far beyond the population bound come only from weights
    // that escaped the branch cutoff (an unequilibrated start); the copy-then-
    // remove loop below would spend ~m steps on them (the reference converts
    // such m to int).  Refuse them instead of running away.
    const double m_limit = 64.0 * static_cast<double>(n_max);
    double m_total = 0.0;
    for (int i = 0; i < n; ++i) {
        const double mw = std::floor(w[i] + rng.uniform());
        m_total += mw > 0.0 ? mw : 0.0;
        if (!(m_total <= m_limit))
            return fail(c, ALEA_ERR_INVALID,
                        "branch multiplicities exceed 64 x (2 target + 1) (walker " + std::to_string(i) +
                            ", weight " + std::to_string(w[i]) + "): equilibrate before branching");
        const int m = static_cast<int>(mw);
        for (int k = 0; k < m; ++k) src.push_back(i);
    }
    if (src.empty()) {
        int best = 0;
        for (int i = 1; i < n; ++i)
            if (w[i] > w[best]) best = i;
        src.push_back(best);
    }
    while (src.size() > n_max) {
        const size_t i = static_cast<size_t>(rng.uniform() * static_cast<double>(src.size()));
        src[i] = src.back();
        src.pop_back();
    }
    while (src.size() < n_min) {
        const size_t i = static_cast<size_t>(rng.uniform() * static_cast<double>(src.size()));
        src.push_back(src[i]);
    }
    // a refused branch leaves the caller's stream where it was, so a retry
    // with more capacity draws the same multiplicities
    if (static_cast<int>(src.size()) > c->capacity)
        return fail(c, ALEA_ERR_NOMEM, "branching exceeded the walker capacity");
    std::memcpy(state, rng.s, 32);
    // genealogy (walker_set.cpp:221-238): ids then parents, one plane each
    std::vector<char> seen(n, 0);
    std::vector<double> idpar(2 * src.size());
    double* nid = idpar.data();
    double* npar = idpar.data() + src.size();
    for (size_t j = 0; j < src.size(); ++j) {
        nid[j] = ids[src[j]];
        npar[j] = par[src[j]];
        if (seen[src[j]]) {
            npar[j] = nid[j];
            nid[j] = c->next_id;
            c->next_id += 1.0;
        } else {
            seen[src[j]] = 1;
        }
    }
    const int nn = static_cast<int>(src.size());
    c->last_src = src;
    // the maps through the pinned stage: ids and parents first, then src
    double* st_idpar = c->h_stage;
    int* st_src = reinterpret_cast<int*>(c->h_stage + 2 * static_cast<size_t>(nn));
    std::memcpy(st_src, src.data(), sizeof(int) * nn);
    CUDA_TRY(c, copy_in(c, c->d_src, st_src, sizeof(int) * nn));
    ++c->launches;
    gather_kernel<<<nn, 256, 0, c->stream>>>(c->rec[1 - c->cur], c->rec[c->cur], c->d_src, nn, c->sys.rec);
    CUDA_TRY(c, cudaGetLastError());
    c->cur = 1 - c->cur;
    c->nw = nn;
    ++c->launches;
    set_scalar_kernel<<<(nn + 255) / 256, 256, 0, c->stream>>>(records(c), nn, c->sys.rec,
                                                                c->sys.o_scal + S_WEIGHT, 1.0);
    CUDA_TRY(c, cudaGetLastError());
    std::memcpy(st_idpar, idpar.data(), 16L * nn);
    CUDA_TRY(c, copy_in(c, c->d_buf, st_idpar, 16L * nn));
    ++c->launches;
    from_soa_kernel<<<(2 * nn + 255) / 256, 256, 0, c->stream>>>(records(c), nn, c->sys.rec, c->sys.o_scal + S_ID,
                                                                  2, c->d_buf);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

int alea_gpu_stream(const alea_gpu_ctx* c, void** stream) {
    if (!c || !stream) return ALEA_ERR_INVALID;
    *stream = static_cast<void*>(c->stream);
    return ALEA_OK;
}

int alea_gpu_transfer_bytes(const alea_gpu_ctx* c, uint64_t* h2d, uint64_t* d2h) {
    if (!c) return ALEA_ERR_INVALID;
    if (h2d) *h2d = c->h2d;
    if (d2h) *d2h = c->d2h;
    return ALEA_OK;
}

int alea_gpu_measure_fp64_peak(int device, double* tflops) {
    if (!tflops) return ALEA_ERR_INVALID;
    *tflops = 0.0;
    return measure_fp64_peak(device, tflops) == cudaSuccess ? ALEA_OK : ALEA_ERR_CUDA;
}

int alea_gpu_launch_count(const alea_gpu_ctx* c, uint64_t* launches) {
    if (!c || !launches) return ALEA_ERR_INVALID;
    *launches = c->launches;
    return ALEA_OK;
}

int alea_gpu_last_kernel_ms(const alea_gpu_ctx* c, double* ms) {
    if (!c || !ms) return ALEA_ERR_INVALID;
    *ms = c->last_ms;
    return ALEA_OK;
}

}  // extern "C"

// ───────────────────────── packed VMC runs ──────────────────────────────
//
// Several contexts' VMC runs stepped together: every step draws each run's
// random numbers and then sweeps the walkers of all runs in one launch per
// sweep body (the one-warp body for the runs that take it, the generic
// 32-thread body for the others), with each run's own system, records and
// parameters (BatchJob).  Per-chain E_L sums of each run reduce on the device
// in walker order and come back in one copy per step, so a run's blocks,
// energy, error and acceptance are those of alea_gpu_vmc_run on its own
// context.  The launch shape of each body (one CTA per walker, or persistent
// CTAs over a work counter, as many as the occupancy calculator allows) is
// picked by timing both on the first steps (PackedTuner); once a step's set
// of runs repeats, the step is captured into a CUDA graph and replayed until
// a run joins or leaves.

namespace {

// A packed run's per-step sums, in alea_gpu_vmc_run's order and rounding:
// state = [step, block, blk[T] (running block sums), e_sum, e2_sum] persists
// on the device across steps.  One thread adds every walker's E_L in walker
// order to its chain's block sum and, in accumulation blocks, to the running
// Σ E_L and Σ E_L² (no contraction, as the host sums); the block sums reset
// when a block starts.  Other threads sum the accepted moves and the largest
// |error flag|.  out = [blk[T], e_sum, e2_sum, Σ accepted, max |error|].
__global__ void run_sums_kernel(const double* records, int nw, long rec, int o_scal, int T, int n_steps,
                                int n_eq, double* state, double* out) {
    if (threadIdx.x == 0) {
        double* blk = state + 2;
        const int step = static_cast<int>(state[0]), block = static_cast<int>(state[1]);
        if (step == 0)
            for (int t = 0; t < T; ++t) blk[t] = 0.0;
        const bool measure = block >= n_eq;
        double e = state[2 + T], e2 = state[3 + T];
        const int base = nw / T, rem = nw % T;
        for (int t = 0; t < T; ++t) {
            const int w0 = t * base + min(t, rem), cnt = base + (t < rem ? 1 : 0);
            double b = blk[t];
            for (int w = w0; w < w0 + cnt; ++w) {
                const double el = records[static_cast<size_t>(w) * rec + o_scal + S_EL];
                b = __dadd_rn(b, el);
                if (measure) {
                    e = __dadd_rn(e, el);
                    e2 = __dadd_rn(e2, __dmul_rn(el, el));
                }
            }
            blk[t] = b;
            out[t] = b;
        }
        state[2 + T] = e;
        state[3 + T] = e2;
        out[T] = e;
        out[T + 1] = e2;
        const int next = step + 1 == n_steps ? 0 : step + 1;
        state[0] = next;
        if (next == 0) state[1] = block + 1;
    }
    __shared__ double red[2][256];
    double na = 0.0, er = 0.0;
    for (int w = threadIdx.x; w < nw; w += blockDim.x) {
        const double* r = records + static_cast<size_t>(w) * rec + o_scal;
        na += r[S_NACC];
        er = fmax(er, fabs(r[S_ERR]));
    }
    red[0][threadIdx.x] = na;
    red[1][threadIdx.x] = er;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            red[0][threadIdx.x] += red[0][threadIdx.x + h];
            red[1][threadIdx.x] = fmax(red[1][threadIdx.x], red[1][threadIdx.x + h]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[T + 2] = red[0][0];
        out[T + 3] = red[1][0];
    }
}

// Body classes of a packed step (kPackedClasses): 0 the one-warp sweep of
// real determinants, 1-3 the generic sweep of 32, 64, 128 threads, 4 the
// one-warp sweep of complex determinants, 5 the one-warp Jastrow-only sweep
// of up to 256 particles.  Each class is one launch on its own stream.
constexpr int kClasses = alea_gpu::kPackedClasses;

// Launch shapes of the packed bodies: for each body class
// the measured time per walker-sweep of shape 0 (one CTA per walker) and
// shape 1 (persistent CTAs); the faster one is kept for the device's
// lifetime (every packed run of the process shares the table).
struct PackedTuner {
    std::mutex mu;
    double ms_per_walker[64][kClasses][2] = {};
    int samples[64][kClasses][2] = {};
    int choice(int dev, int body) {
        std::lock_guard<std::mutex> lk(mu);
        for (int shape = 0; shape < 2; ++shape)
            if (samples[dev][body][shape] < 2) return shape;   // still measuring
        return ms_per_walker[dev][body][1] < ms_per_walker[dev][body][0] ? 1 : 0;
    }
    bool settled(int dev, int body) {
        std::lock_guard<std::mutex> lk(mu);
        return samples[dev][body][0] >= 2 && samples[dev][body][1] >= 2;
    }
    void record(int dev, int body, int shape, double ms_per_w) {
        std::lock_guard<std::mutex> lk(mu);
        int& n = samples[dev][body][shape];
        double& m = ms_per_walker[dev][body][shape];
        m = (m * n + ms_per_w) / (n + 1);
        ++n;
    }
};
PackedTuner g_packed_tuner;

struct PackedRunState {
    alea_gpu_ctx* c = nullptr;
    alea_gpu_run_config cfg{};
    int T = 1;
    int block = 0, step = 0;
    int cls = 0;                   // body class (kClasses)
    size_t smem = 0;
    size_t stats_off = 0;
    double* d_state = nullptr;     // run_sums_kernel's [step, block, blk[T], e_sum, e2_sum]
    std::vector<std::vector<double>> chain;
    std::vector<double> blk;
    std::vector<int64_t> blk_n;
    double e_sum = 0.0, e2_sum = 0.0;
    int64_t n_tot = 0, acc = 0, prop = 0, moves = 0, evals = 0;
    std::chrono::steady_clock::time_point t0;
    bool done = false;
    int status = ALEA_OK;
    alea_gpu_run_result res{};
    std::vector<double> blocks;
};

}  // namespace

struct alea_gpu_packed {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<PackedRunState> runs;
    bool dirty = true;
    BatchJob* d_jobs = nullptr;
    BatchJob* h_jobs = nullptr;   // pinned
    int jobs_cap = 0;
    double* d_stats = nullptr;
    double* h_stats = nullptr;    // pinned
    size_t stats_cap = 0;
    int* d_next = nullptr;         // one work counter per class
    int n_jobs[kClasses] = {}, job0[kClasses] = {}, total[kClasses] = {};
    size_t smem[kClasses] = {};
    cudaStream_t cls_stream[kClasses] = {};
    cudaEvent_t fork = nullptr, join[kClasses] = {};
    cudaGraphExec_t graph = nullptr;
    int graph_shapes[kClasses] = {-1, -1, -1, -1, -1, -1};
    cudaEvent_t ev[2 * kClasses] = {};
    std::string err;
    uint64_t launches = 0;
};

namespace {

int pfail(alea_gpu_packed* P, int code, const std::string& msg) {
    P->err = msg;
    return code;
}

#define PCUDA(P, expr)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return pfail((P), ALEA_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void packed_drop_graph(alea_gpu_packed* P) {
    if (P->graph) cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
}

// Job tables, stats slots and the shared-memory reservation of the runs still
// going, after one joined or left.
int packed_rebuild(alea_gpu_packed* P) {
    packed_drop_graph(P);
    std::vector<BatchJob> lists[kClasses];
    size_t stats = 0;
    for (int k = 0; k < kClasses; ++k) P->smem[k] = 0, P->total[k] = 0;
    for (PackedRunState& r : P->runs) {
        if (r.done) continue;
        alea_gpu_ctx* c = r.c;
        if (int rc = ensure_randoms(c, r.cfg.n_substeps)) return pfail(P, rc, c->err);
        if (int rc = set_sigma(c, r.cfg.tau)) return pfail(P, rc, c->err);
        if (!c->d_sys) PCUDA(P, cudaMallocAsync(&c->d_sys, sizeof(DevSys), c->stream));
        PCUDA(P, cudaMemcpyAsync(c->d_sys, &c->sys, sizeof(DevSys), cudaMemcpyHostToDevice, c->stream));
        if (!r.d_state) {
            PCUDA(P, cudaMallocAsync(&r.d_state, 8 * (static_cast<size_t>(r.T) + 4), c->stream));
            PCUDA(P, cudaMemsetAsync(r.d_state, 0, 8 * (static_cast<size_t>(r.T) + 4), c->stream));
        }
        PCUDA(P, cudaStreamSynchronize(c->stream));
        BatchJob j{};
        j.sys = c->d_sys;
        j.records = records(c);
        j.randoms = c->randoms;
        j.stride = c->nw;
        j.prm.mode = 0;
        j.prm.n_sub = r.cfg.n_substeps;
        j.prm.drift = r.cfg.use_drift;
        j.prm.tau = r.cfg.tau;
        j.prm.sigma = c->d_sigma;
        j.pairs = c->pairs;
        j.npair = c->npair;
        j.nw = c->nw;
        j.first = P->total[r.cls];
        P->total[r.cls] += c->nw;
        lists[r.cls].push_back(j);
        P->smem[r.cls] = std::max(P->smem[r.cls], r.smem);
        r.stats_off = stats;
        stats += static_cast<size_t>(r.T) + 4;
    }
    int need = 0;
    for (int k = 0; k < kClasses; ++k) {
        P->job0[k] = need;
        P->n_jobs[k] = static_cast<int>(lists[k].size());
        need += P->n_jobs[k];
    }
    if (need > P->jobs_cap) {
        if (P->d_jobs) cudaFreeAsync(P->d_jobs, P->stream);
        if (P->h_jobs) cudaFreeHost(P->h_jobs);
        P->d_jobs = nullptr;
        P->h_jobs = nullptr;
        const int cap = std::max(need, 2 * P->jobs_cap);
        PCUDA(P, cudaMallocAsync(&P->d_jobs, sizeof(BatchJob) * cap, P->stream));
        PCUDA(P, cudaMallocHost(&P->h_jobs, sizeof(BatchJob) * cap));
        P->jobs_cap = cap;
    }
    if (stats > P->stats_cap) {
        if (P->d_stats) cudaFreeAsync(P->d_stats, P->stream);
        if (P->h_stats) cudaFreeHost(P->h_stats);
        P->d_stats = nullptr;
        P->h_stats = nullptr;
        const size_t cap = std::max(stats, 2 * P->stats_cap);
        PCUDA(P, cudaMallocAsync(&P->d_stats, 8 * cap, P->stream));
        PCUDA(P, cudaMallocHost(&P->h_stats, 8 * cap));
        P->stats_cap = cap;
    }
    if (!P->d_next) PCUDA(P, cudaMallocAsync(&P->d_next, kClasses * sizeof(int), P->stream));
    for (int k = 0; k < kClasses; ++k) std::copy(lists[k].begin(), lists[k].end(), P->h_jobs + P->job0[k]);
    if (need) PCUDA(P, cudaMemcpyAsync(P->d_jobs, P->h_jobs, sizeof(BatchJob) * need, cudaMemcpyHostToDevice,
                                       P->stream));
    PCUDA(P, cudaStreamSynchronize(P->stream));
    PCUDA(P, reserve_smem(*std::max_element(P->smem, P->smem + kClasses)));
    P->dirty = false;
    return ALEA_OK;
}

bool packed_zero_energy(const alea_gpu_packed* P, int cls) {
    for (const PackedRunState& r : P->runs)
        if (!r.done && r.cls == cls)
            for (int t = 0; t < r.c->sys.nterms; ++t)
                if (r.c->sys.terms[t].kind == 2) return true;
    return false;
}

// Grid of a packed launch of class k: every walker its CTA (shape 0), or as
// many persistent CTAs as are resident on the device at once (shape 1).
int packed_grid(alea_gpu_packed* P, int k, int shape) {
    const int total = P->total[k];
    if (shape == 0) return total;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, P->device);
    const int per_sm = k == 5                ? boson_batch_ctas_per_sm(P->smem[k])
                       : (k == 0 || k == 4) ? fast_batch_ctas_per_sm(k == 4, P->smem[k])
                                            : batch_ctas_per_sm(16 << k, P->smem[k]);
    return std::max(1, std::min(total, sms * per_sm));
}

// The launches of one step: draws, then the classes' packed sweeps on their
// own streams (forked from and joined back into the engine's stream, so they
// run side by side), then the per-run sums and their copy.
int packed_enqueue(alea_gpu_packed* P, const int shape[kClasses], bool timed) {
    for (const PackedRunState& r : P->runs) {
        if (r.done) continue;
        alea_gpu_ctx* c = r.c;
        const int nt = std::min(c->n_streams, c->nw);
        draw_kernel<<<(nt + 127) / 128, 128, 0, P->stream>>>(c->streams, c->n_streams, c->nw, c->sys.np, c->nw,
                                                             r.cfg.n_substeps, c->sys.zk, c->sys.zw, c->sys.zf,
                                                             c->sys.zr, c->randoms, c->sys.dim);
        ++P->launches;
    }
    PCUDA(P, cudaGetLastError());
    PCUDA(P, cudaMemsetAsync(P->d_next, 0, kClasses * sizeof(int), P->stream));
    PCUDA(P, cudaEventRecord(P->fork, P->stream));
    for (int k = 0; k < kClasses; ++k) {
        if (!P->n_jobs[k]) continue;
        cudaStream_t st = P->cls_stream[k];
        PCUDA(P, cudaStreamWaitEvent(st, P->fork, 0));
        if (timed) PCUDA(P, cudaEventRecord(P->ev[2 * k], st));
        const BatchJob* jobs = P->d_jobs + P->job0[k];
        if (k == 5)
            PCUDA(P, launch_sweep_boson_batch(packed_zero_energy(P, 5), jobs, P->n_jobs[k], P->total[k],
                                              packed_grid(P, k, shape[k]), P->smem[k], P->d_next + k, st));
        else if (k == 0 || k == 4)
            PCUDA(P, launch_sweep_fast_batch(k == 0 && packed_zero_energy(P, 0), k == 4, jobs, P->n_jobs[k],
                                             P->total[k], packed_grid(P, k, shape[k]), P->smem[k], P->d_next + k,
                                             st));
        else
            PCUDA(P, launch_sweep_generic_batch(16 << k, jobs, P->n_jobs[k], P->total[k],
                                                packed_grid(P, k, shape[k]), P->smem[k], P->d_next + k, st));
        ++P->launches;
        if (timed) PCUDA(P, cudaEventRecord(P->ev[2 * k + 1], st));
        PCUDA(P, cudaEventRecord(P->join[k], st));
        PCUDA(P, cudaStreamWaitEvent(P->stream, P->join[k], 0));
    }
    for (const PackedRunState& r : P->runs) {
        if (r.done) continue;
        alea_gpu_ctx* c = r.c;
        run_sums_kernel<<<1, 256, 0, P->stream>>>(records(c), c->nw, c->sys.rec, c->sys.o_scal, r.T,
                                                  r.cfg.n_steps, r.cfg.n_equilibration_blocks, r.d_state,
                                                  P->d_stats + r.stats_off);
        ++P->launches;
    }
    PCUDA(P, cudaGetLastError());
    size_t n = 0;
    for (const PackedRunState& r : P->runs)
        if (!r.done) n = std::max(n, r.stats_off + static_cast<size_t>(r.T) + 4);
    PCUDA(P, cudaMemcpyAsync(P->h_stats, P->d_stats, 8 * n, cudaMemcpyDeviceToHost, P->stream));
    return ALEA_OK;
}

// The run's result from its blocks, as alea_gpu_vmc_run forms it.
void packed_finish(PackedRunState& r) {
    if (r.d_state) cudaFreeAsync(r.d_state, r.c->stream);
    r.d_state = nullptr;
    for (int t = 0; t < r.T; ++t) r.blocks.insert(r.blocks.end(), r.chain[t].begin(), r.chain[t].end());
    double mean = 0.0, err = 0.0;
    reblock(r.blocks, mean, err);
    r.res.energy = mean;
    r.res.energy_error = err;
    const double m = r.n_tot ? r.e_sum / static_cast<double>(r.n_tot) : 0.0;
    r.res.variance = r.n_tot ? r.e2_sum / static_cast<double>(r.n_tot) - m * m : 0.0;
    r.res.acceptance = r.prop ? static_cast<double>(r.acc) / static_cast<double>(r.prop) : 0.0;
    r.res.walltime_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - r.t0).count();
    r.res.n_walkers = r.c->nw;
    r.res.e_trial = 0.0;
    r.res.n_moves = r.moves;
    r.res.n_evaluations = r.evals;
    r.done = true;
}

}  // namespace

namespace alea_gpu {

int packed_create(int device, alea_gpu_packed** out) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return ALEA_ERR_CUDA;
    auto* P = new alea_gpu_packed();
    P->device = device;
    bool ok = cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaStream_t& st : P->cls_stream) ok = ok && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
    for (cudaEvent_t& e : P->ev) ok = ok && cudaEventCreate(&e) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming) == cudaSuccess;
    for (cudaEvent_t& e : P->join) ok = ok && cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        packed_destroy(P);
        return ALEA_ERR_CUDA;
    }
    *out = P;
    return ALEA_OK;
}

void packed_destroy(alea_gpu_packed* P) {
    if (!P) return;
    cudaSetDevice(P->device);
    packed_drop_graph(P);
    for (PackedRunState& r : P->runs)
        if (r.d_state) cudaFreeAsync(r.d_state, P->stream);
    if (P->stream) {
        for (void* p : {static_cast<void*>(P->d_jobs), static_cast<void*>(P->d_stats), static_cast<void*>(P->d_next)})
            if (p) cudaFreeAsync(p, P->stream);
        cudaStreamSynchronize(P->stream);
        cudaStreamDestroy(P->stream);
    }
    if (P->h_jobs) cudaFreeHost(P->h_jobs);
    if (P->h_stats) cudaFreeHost(P->h_stats);
    for (cudaEvent_t e : P->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : P->join)
        if (e) cudaEventDestroy(e);
    if (P->fork) cudaEventDestroy(P->fork);
    for (cudaStream_t st : P->cls_stream)
        if (st) cudaStreamDestroy(st);
    delete P;
}

const std::string& packed_error(const alea_gpu_packed* P) { return P->err; }

int packed_class(const alea_gpu_ctx* c) {
    const char* e = std::getenv("ALEA_GPU_SWEEP");
    const bool one_warp = e == nullptr || std::strcmp(e, "generic") != 0;
    if (one_warp && c->nt == 32 && fast_sweep_eligible(c->sys)) return c->sys.cplx ? 4 : 0;
    if (one_warp && boson_sweep_eligible(c->sys)) return 5;
    return c->nt == 32 ? 1 : c->nt == 64 ? 2 : 3;
}

// A context (walkers uploaded, FP64) joins with its VMC run; its random
// streams are set as alea_gpu_vmc_run sets them.  Returns the run's slot.
int packed_add(alea_gpu_packed* P, alea_gpu_ctx* c, const alea_gpu_run_config& cfg, int* slot) {
    if (!P || !c || c->device != P->device) return pfail(P, ALEA_ERR_INVALID, "packed run: context on another device");
    if (c->sys.f32) return pfail(P, ALEA_ERR_UNSUPPORTED, "packed run: FP64 contexts only");
    if (c->sys.dim != 2) return pfail(P, ALEA_ERR_UNSUPPORTED, "packed run: two-dimensional systems only");
    if (c->nw < 1 || cfg.n_steps < 1 || cfg.n_substeps < 1 || cfg.n_accumulation_blocks < 0 ||
        cfg.n_equilibration_blocks < 0)
        return pfail(P, ALEA_ERR_INVALID, "packed run: empty population or bad run configuration");
    PackedRunState r;
    r.c = c;
    r.cfg = cfg;
    r.T = std::min(std::max(cfg.n_streams, 1), c->nw);
    if (int rc = alea_gpu_set_streams(c, cfg.seed, ALEA_STREAM_VMC, r.T)) return pfail(P, rc, c->err);
    r.cls = packed_class(c);
    const bool fast = r.cls == 0 || r.cls == 4 || r.cls == 5;
    r.smem = fast ? static_cast<size_t>(c->sys.f_total) * 8 : c->smem;
    r.chain.assign(r.T, {});
    r.blk.assign(r.T, 0.0);
    r.blk_n.assign(r.T, 0);
    r.t0 = std::chrono::steady_clock::now();
    if (cfg.n_equilibration_blocks + cfg.n_accumulation_blocks == 0) r.done = true;
    if (slot) *slot = static_cast<int>(P->runs.size());
    P->runs.push_back(std::move(r));
    P->dirty = true;
    return ALEA_OK;
}

int packed_active(const alea_gpu_packed* P) {
    int n = 0;
    for (const PackedRunState& r : P->runs) n += r.done ? 0 : 1;
    return n;
}

bool packed_done(const alea_gpu_packed* P, int slot, int* status, alea_gpu_run_result* res) {
    const PackedRunState& r = P->runs[slot];
    if (!r.done) return false;
    if (status) *status = r.status;
    if (res) *res = r.res;
    return true;
}

const std::vector<double>& packed_blocks(const alea_gpu_packed* P, int slot) { return P->runs[slot].blocks; }

// Stop run `slot` before its next step (status ALEA_ERR_CANCELLED).
void packed_cancel(alea_gpu_packed* P, int slot) {
    PackedRunState& r = P->runs[slot];
    if (r.done) return;
    r.status = ALEA_ERR_CANCELLED;
    r.done = true;
    P->dirty = true;
}

// Forget finished runs (their contexts are the caller's); slots renumber.
void packed_prune(alea_gpu_packed* P) {
    std::vector<PackedRunState> keep;
    for (PackedRunState& r : P->runs) {
        if (!r.done) {
            keep.push_back(std::move(r));
        } else if (r.d_state) {
            cudaFreeAsync(r.d_state, P->stream);
            r.d_state = nullptr;
        }
    }
    P->runs.swap(keep);
    P->dirty = true;
}

// One step of every run still going.
int packed_step(alea_gpu_packed* P) {
    if (packed_active(P) == 0) return ALEA_OK;
    PCUDA(P, cudaSetDevice(P->device));
    if (P->dirty)
        if (int rc = packed_rebuild(P)) return rc;
    const int dev = P->device;
    int shape[kClasses];
    bool settled = true;
    for (int k = 0; k < kClasses; ++k) {
        shape[k] = g_packed_tuner.choice(dev, k);
        if (P->n_jobs[k] && !g_packed_tuner.settled(dev, k)) settled = false;
    }
    if (settled) {
        bool same = P->graph != nullptr;
        for (int k = 0; k < kClasses && same; ++k) same = P->graph_shapes[k] == shape[k];
        if (!same) packed_drop_graph(P);
        if (!P->graph) {
            cudaGraph_t g = nullptr;
            PCUDA(P, cudaStreamBeginCapture(P->stream, cudaStreamCaptureModeThreadLocal));
            const int rc = packed_enqueue(P, shape, false);
            const cudaError_t ce = cudaStreamEndCapture(P->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            PCUDA(P, ce);
            const cudaError_t ie = cudaGraphInstantiate(&P->graph, g, 0);
            cudaGraphDestroy(g);
            PCUDA(P, ie);
            for (int k = 0; k < kClasses; ++k) P->graph_shapes[k] = shape[k];
        }
        PCUDA(P, cudaGraphLaunch(P->graph, P->stream));
    } else {
        if (int rc = packed_enqueue(P, shape, true)) return rc;
    }
    PCUDA(P, cudaStreamSynchronize(P->stream));
    if (!settled) {
        for (int k = 0; k < kClasses; ++k) {
            float ms = 0.f;
            if (P->n_jobs[k] && cudaEventElapsedTime(&ms, P->ev[2 * k], P->ev[2 * k + 1]) == cudaSuccess)
                g_packed_tuner.record(dev, k, shape[k], ms / P->total[k]);
        }
    }
    for (PackedRunState& r : P->runs) {
        if (r.done) continue;
        alea_gpu_ctx* c = r.c;
        const double* st = P->h_stats + r.stats_off;
        c->launches += 3;
        if (st[r.T + 3] != 0.0) {
            r.status = fail(c, ALEA_ERR_SINGULAR, "a walker's accepted determinant is singular or nonfinite");
            r.done = true;
            P->dirty = true;
            continue;
        }
        const int64_t proposed = static_cast<int64_t>(r.cfg.n_substeps) * c->sys.np * c->nw;
        r.moves += proposed;
        r.evals += c->nw;
        const bool measure = r.block >= r.cfg.n_equilibration_blocks;
        if (measure) {
            const int base = c->nw / r.T, rem = c->nw % r.T;
            for (int t = 0; t < r.T; ++t) {
                r.blk[t] = st[t];
                r.blk_n[t] += base + (t < rem ? 1 : 0);
            }
            r.n_tot += c->nw;
            r.e_sum = st[r.T];
            r.e2_sum = st[r.T + 1];
            r.acc += static_cast<int64_t>(st[r.T + 2]);
            r.prop += proposed;
        }
        if (++r.step == r.cfg.n_steps) {
            if (measure)
                for (int t = 0; t < r.T; ++t) r.chain[t].push_back(r.blk[t] / static_cast<double>(r.blk_n[t]));
            std::fill(r.blk.begin(), r.blk.end(), 0.0);
            std::fill(r.blk_n.begin(), r.blk_n.end(), 0);
            r.step = 0;
            if (++r.block == r.cfg.n_equilibration_blocks + r.cfg.n_accumulation_blocks) {
                packed_finish(r);
                P->dirty = true;
            }
        }
    }
    return ALEA_OK;
}

uint64_t packed_launches(const alea_gpu_packed* P) { return P->launches; }

}  // namespace alea_gpu

extern "C" int alea_gpu_vmc_run_packed(alea_gpu_ctx* const* ctxs, int n, const alea_gpu_run_config* cfgs,
                                       alea_gpu_run_result* results, int* statuses) {
    if (!ctxs || n < 1 || !cfgs || !results) return ALEA_ERR_INVALID;
    alea_gpu_packed* P = nullptr;
    if (int rc = alea_gpu::packed_create(ctxs[0]->device, &P)) return rc;
    int rc = ALEA_OK;
    for (int i = 0; i < n && rc == ALEA_OK; ++i) {
        if (!ctxs[i]) rc = ALEA_ERR_INVALID;
        else rc = alea_gpu::packed_add(P, ctxs[i], cfgs[i], nullptr);
        if (rc) g_create_error = P->err;
    }
    while (rc == ALEA_OK && alea_gpu::packed_active(P) > 0) {
        rc = alea_gpu::packed_step(P);
        if (rc) g_create_error = P->err;
    }
    for (int i = 0; i < n && rc == ALEA_OK; ++i) {
        int st = ALEA_OK;
        alea_gpu::packed_done(P, i, &st, &results[i]);
        if (statuses) statuses[i] = st;
    }
    alea_gpu::packed_destroy(P);
    return rc;
}

extern "C" {

// ───────────────────────── forward walking ─────────────────────────────

namespace {

void fw_free_run(alea_gpu_ctx* c) {
    FwState* f = c->fw;
    if (!f) return;
    for (FwSlot& sl : f->slots)
        if (sl.d_pos) cudaFreeAsync(sl.d_pos, c->stream);
    f->slots.clear();
    for (void* p : {static_cast<void*>(f->d_idx), static_cast<void*>(f->d_kw), static_cast<void*>(f->d_v)})
        if (p) cudaFreeAsync(p, c->stream);
    f->d_idx = nullptr;
    f->d_kw = f->d_v = nullptr;
}

void fw_free(alea_gpu_ctx* c) {
    if (!c->fw) return;
    fw_free_run(c);
    for (EstimatorSet*& e : c->fw->est) est_free(e, c->stream);
    delete c->fw;
    c->fw = nullptr;
}

// DMC::DMC's forward-walking checks and ForwardWalking::prepare
// (src/qmc/dmc.cpp:102-138, :591-600; src/qmc/forward_walking.cpp:49-73):
// lags in whole steps of τ·n_substeps, the largest inside the equilibration,
// the interval dividing the steps per block; a ring of max_lag/interval + 1
// snapshots of the population capacity.
int fw_prepare(alea_gpu_ctx* c, const alea_gpu_run_config* cfg) {
    FwState* f = c->fw;
    if (!f) return ALEA_OK;
    fw_free_run(c);
    const double step_time = cfg->tau * static_cast<double>(cfg->n_substeps);
    if (!(std::isfinite(step_time) && step_time > 0.0))
        return fail(c, ALEA_ERR_INVALID, "dmc: forward walking needs time_step > 0 and sub_steps >= 1");
    if (f->interval < 1 || cfg->n_steps <= 0 || cfg->n_steps % f->interval != 0)
        return fail(c, ALEA_ERR_INVALID, "dmc: forward_walking interval (" + std::to_string(f->interval) +
                                             ") must be >= 1 and divide steps_per_block (" +
                                             std::to_string(cfg->n_steps) + ")");
    f->lag_steps.clear();
    for (double lag : f->lags) {
        const double steps = lag / step_time, whole = std::round(steps);
        if (std::abs(steps - whole) > 1e-9 * std::max(1.0, steps))
            return fail(c, ALEA_ERR_INVALID, "dmc: forward_walking lag " + std::to_string(lag) +
                                                 " is not a whole number of steps of time_step * sub_steps = " +
                                                 std::to_string(step_time));
        f->lag_steps.push_back(static_cast<long>(whole));
    }
    const long eq_steps = static_cast<long>(std::max(0, cfg->n_equilibration_blocks)) * cfg->n_steps;
    const long max_lag = f->lag_steps.back();
    if (max_lag > eq_steps)
        return fail(c, ALEA_ERR_INVALID, "dmc: the largest forward_walking lag (" + std::to_string(max_lag) +
                                             " steps) exceeds the equilibration (" + std::to_string(eq_steps) +
                                             " steps): snapshots start that many steps before accumulation");
    f->step_time = step_time;
    f->first_measured = eq_steps;
    f->first_snapshot = eq_steps - max_lag;
    const size_t n = f->lags.size();
    f->blk_wpot.assign(n, 0.0);
    f->blk_w.assign(n, 0.0);
    f->block_pot.assign(n, {});
    f->measurements.assign(n, 0);
    f->surviving.assign(n, 0.0);
    f->slots.assign(static_cast<size_t>(max_lag / f->interval + 1), FwSlot{});
    const size_t cap = static_cast<size_t>(c->capacity);
    for (FwSlot& sl : f->slots)
        if (cudaMallocAsync(&sl.d_pos, cap * c->sys.np * 2 * 8, c->stream) != cudaSuccess)
            return fail(c, ALEA_ERR_NOMEM, "forward walking: snapshot allocation failed");
    if (cudaMallocAsync(&f->d_idx, cap * sizeof(int), c->stream) != cudaSuccess ||
        cudaMallocAsync(&f->d_kw, cap * 8, c->stream) != cudaSuccess ||
        cudaMallocAsync(&f->d_v, cap * 8, c->stream) != cudaSuccess)
        return fail(c, ALEA_ERR_NOMEM, "forward walking: allocation failed");
    for (EstimatorSet* e : f->est) {
        std::string err;
        if (int rc = est_reset(e, c->stream, err)) return fail(c, rc, err);
    }
    return ALEA_OK;
}

bool fw_snapshot_step(const FwState* f, long step) {
    return step >= f->first_snapshot && (step - f->first_snapshot) % f->interval == 0;
}

size_t fw_slot_of(const FwState* f, long step) {
    return static_cast<size_t>((step - f->first_snapshot) / f->interval) % f->slots.size();
}

// ForwardWalking::measure (forward_walking.cpp:133-173): descendant weights
// D[a] = Σ_{w: a(w)=a} W_w in walker order, the ancestors with D > 0 in
// snapshot order measured with weights D: the lag's estimators and the
// potential energy (Σ D V / Σ D into the block).
int fw_measure(alea_gpu_ctx* c, size_t lag, const FwSlot& sl) {
    FwState* f = c->fw;
    std::vector<double> w;
    if (int rc = read_scalars(c, S_WEIGHT, w)) return rc;
    if (sl.anc.size() != w.size())
        return fail(c, ALEA_ERR_INVALID, "forward walking: ancestry out of step with the population");
    std::vector<double> dw(static_cast<size_t>(sl.nw), 0.0);
    for (size_t i = 0; i < w.size(); ++i) dw[sl.anc[i]] += w[i];
    std::vector<int> kept;
    std::vector<double> kw;
    for (int a = 0; a < sl.nw; ++a)
        if (dw[a] > 0.0) {
            kept.push_back(a);
            kw.push_back(dw[a]);
        }
    if (kept.empty()) return ALEA_OK;
    const int nk = static_cast<int>(kept.size());
    CUDA_TRY(c, copy_in(c, f->d_idx, kept.data(), sizeof(int) * nk));
    CUDA_TRY(c, copy_in(c, f->d_kw, kw.data(), 8L * nk));
    ++c->launches;
    CUDA_TRY(c, launch_potential(c->nt, nk, c->smem, c->stream, c->sys, sl.d_pos, f->d_idx, c->pairs, c->npair,
                                 f->d_v));
    const EstSource src{sl.d_pos, static_cast<long>(c->sys.np) * 2, 0, -1, f->d_idx, nk};
    std::string err;
    if (int rc = est_accumulate(f->est[lag], c->sys, src, f->d_kw, false, 1, c->pairs, c->npair, c->stream, err,
                                &c->launches))
        return fail(c, rc, err);
    std::vector<double> v(static_cast<size_t>(nk));
    CUDA_TRY(c, copy_out(c, v.data(), f->d_v, 8L * nk));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    double weighted = 0.0, total = 0.0;
    for (int k = 0; k < nk; ++k) {
        weighted += kw[k] * v[k];
        total += kw[k];
    }
    f->blk_wpot[lag] += weighted;
    f->blk_w[lag] += total;
    ++f->measurements[lag];
    f->surviving[lag] += static_cast<double>(nk) / static_cast<double>(sl.nw);
    return ALEA_OK;
}

// ForwardWalking::observe (forward_walking.cpp:113-131): after the step's
// moves and reweighting, before the branch.
int fw_observe(alea_gpu_ctx* c, long step) {
    FwState* f = c->fw;
    if (!f) return ALEA_OK;
    const Phase phase("alea.forward_walking");
    if (fw_snapshot_step(f, step)) {
        FwSlot& sl = f->slots[fw_slot_of(f, step)];
        sl.step = step;
        sl.nw = c->nw;
        const int n = c->sys.np * 2;
        const long tot = static_cast<long>(n) * c->nw;
        ++c->launches;
        to_rows_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, c->stream>>>(records(c), c->nw, c->sys.rec,
                                                                                  c->sys.o_pos, n, sl.d_pos);
        CUDA_TRY(c, cudaGetLastError());
        sl.anc.resize(static_cast<size_t>(c->nw));
        for (int i = 0; i < c->nw; ++i) sl.anc[i] = i;
    }
    if (step < f->first_measured) return ALEA_OK;
    for (size_t i = 0; i < f->lag_steps.size(); ++i) {
        const long taken = step - f->lag_steps[i];
        if (taken < f->first_snapshot || !fw_snapshot_step(f, taken)) continue;
        const FwSlot& sl = f->slots[fw_slot_of(f, taken)];
        if (sl.step != taken) return fail(c, ALEA_ERR_INVALID, "forward walking: snapshot ring overwritten too early");
        if (int rc = fw_measure(c, i, sl)) return rc;
    }
    return ALEA_OK;
}

// ForwardWalking::branch (forward_walking.cpp:175-182).
void fw_branch(alea_gpu_ctx* c) {
    if (!c->fw) return;
    for (FwSlot& sl : c->fw->slots) {
        if (sl.step < 0) continue;
        std::vector<int> g(c->last_src.size());
        for (size_t j = 0; j < g.size(); ++j) g[j] = sl.anc[c->last_src[j]];
        sl.anc.swap(g);
    }
}

int fw_start_block(alea_gpu_ctx* c) {
    FwState* f = c->fw;
    if (!f) return ALEA_OK;
    std::fill(f->blk_wpot.begin(), f->blk_wpot.end(), 0.0);
    std::fill(f->blk_w.begin(), f->blk_w.end(), 0.0);
    for (EstimatorSet* e : f->est) {
        std::string err;
        if (int rc = est_start_block(e, c->stream, err)) return fail(c, rc, err);
    }
    return ALEA_OK;
}

int fw_stop_block(alea_gpu_ctx* c) {
    FwState* f = c->fw;
    if (!f) return ALEA_OK;
    for (size_t i = 0; i < f->lags.size(); ++i) {
        if (f->blk_w[i] > 0.0) f->block_pot[i].push_back(f->blk_wpot[i] / f->blk_w[i]);
        std::string err;
        // a lag with no measurement in the block (none possible) closes nothing
        if (est_count(f->est[i]) > 0 && f->measurements[i] > 0)
            if (int rc = est_stop_block(f->est[i], c->stream, err, &c->d2h)) return fail(c, rc, err);
    }
    return ALEA_OK;
}

}  // namespace

// ───────────────────────── configurations / carry-over ────────────────

namespace {

// Fresh walkers from n_rows AoS rows already on c's device (walker w takes
// row w mod n_rows): what alea_gpu_upload_walkers does with SoA positions.
int fresh_walkers(alea_gpu_ctx* c, const double* d_rows, int n_rows, int nw) {
    const DevSys& s = c->sys;
    c->cur = 0;
    c->nw = nw;
    CUDA_TRY(c, cudaMemsetAsync(records(c), 0, static_cast<size_t>(s.rec) * 8 * nw, c->stream));
    const long n = static_cast<long>(s.np) * s.dim * nw;
    ++c->launches;
    from_rows_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, c->stream>>>(records(c), nw, s.rec, s.o_pos,
                                                                              s.np * s.dim, d_rows, n_rows);
    ++c->launches;
    set_scalar_kernel<<<(nw + 255) / 256, 256, 0, c->stream>>>(records(c), nw, s.rec, s.o_scal + S_WEIGHT, 1.0);
    CUDA_TRY(c, cudaGetLastError());
    c->next_id = 1.0;
    return launch_evaluate(c);
}

}  // namespace

int alea_gpu_set_checkpoint_hook(alea_gpu_ctx* c, alea_gpu_checkpoint_fn fn, void* user) {
    if (!c) return ALEA_ERR_INVALID;
    c->ckpt_fn = fn;
    c->ckpt_user = user;
    return ALEA_OK;
}

int alea_gpu_final_configurations(alea_gpu_ctx* c, double* rows, int* nw) {
    if (!c || !nw) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    *nw = c->nw;
    if (!rows || c->nw == 0) return ALEA_OK;
    const int n = c->sys.np * c->sys.dim;
    const long tot = static_cast<long>(n) * c->nw;
    ++c->launches;
    to_rows_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, c->stream>>>(records(c), c->nw, c->sys.rec,
                                                                              c->sys.o_pos, n, c->d_buf);
    CUDA_TRY(c, cudaGetLastError());
    CUDA_TRY(c, copy_out(c, rows, c->d_buf, static_cast<size_t>(tot) * 8));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

int alea_gpu_seed_walker_rows(alea_gpu_ctx* c, const double* rows, int n_rows, int nw) {
    if (!c) return ALEA_ERR_INVALID;
    if (!rows || n_rows < 1) return fail(c, ALEA_ERR_INVALID, "seed_walker_rows: no configurations to seed from");
    if (nw < 1 || nw > c->capacity) return fail(c, ALEA_ERR_NOMEM, "walker count exceeds the capacity");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const int used = std::min(n_rows, nw);
    for (long i = 0, n = static_cast<long>(used) * c->sys.np * c->sys.dim; i < n; ++i)
        if (!std::isfinite(rows[i]))
            return fail(c, ALEA_ERR_INVALID, "configuration rows must be finite (entry " + std::to_string(i) + ")");
    CUDA_TRY(c, copy_in(c, c->d_buf, rows, static_cast<size_t>(used) * c->sys.np * c->sys.dim * 8));
    return fresh_walkers(c, c->d_buf, used, nw);
}

int alea_gpu_carry_over(alea_gpu_ctx* from, alea_gpu_ctx* to, int nw, int mode) {
    if (!from || !to || from == to) return ALEA_ERR_INVALID;
    if (mode != ALEA_CARRY_POSITIONS && mode != ALEA_CARRY_STATE)
        return fail(to, ALEA_ERR_INVALID, "carry_over: unknown mode");
    if (nw < 1 || nw > to->capacity) return fail(to, ALEA_ERR_NOMEM, "walker count exceeds the capacity");
    if (from->nw < 1) return fail(to, ALEA_ERR_INVALID, "carry_over: the source context has no walkers");
    if (from->sys.np != to->sys.np || from->sys.dim != to->sys.dim)
        return fail(to, ALEA_ERR_INVALID, "carry_over: particle counts or dimensions differ");
    const int used = std::min(from->nw, nw);
    const bool peer = from->device != to->device;
    if (mode == ALEA_CARRY_STATE) {
        if (from->fingerprint != to->fingerprint)
            return fail(to, ALEA_ERR_INVALID,
                        "carry_over: the contexts were created from different systems; carry positions instead");
        if (from->sys.f32 != to->sys.f32)
            return fail(to, ALEA_ERR_INVALID, "carry_over: the contexts run at different precisions");
        const DevSys& s = to->sys;
        CUDA_TRY(to, cudaSetDevice(from->device));
        CUDA_TRY(to, cudaStreamSynchronize(from->stream));
        const double* src = from->rec[from->cur];
        CUDA_TRY(to, cudaSetDevice(to->device));
        if (peer) {   // stage the used records in the destination's spare buffer
            double* stage = to->rec[1 - to->cur];
            CUDA_TRY(to, cudaMemcpyPeerAsync(stage, to->device, src, from->device,
                                             static_cast<size_t>(used) * s.rec * 8, to->stream));
            src = stage;
        }
        ++to->launches;
        cycle_index_kernel<<<(nw + 255) / 256, 256, 0, to->stream>>>(to->d_src, nw, used);
        ++to->launches;
        gather_kernel<<<nw, 256, 0, to->stream>>>(to->rec[to->cur], src, to->d_src, nw, s.rec);
        // a fresh ensemble: weight 1, no age, no ancestry, no displacement sums
        to->launches += 6;
        set_scalar_kernel<<<(nw + 255) / 256, 256, 0, to->stream>>>(to->rec[to->cur], nw, s.rec,
                                                                     s.o_scal + S_WEIGHT, 1.0);
        for (int slot : {S_RRP, S_RRA, S_AGE, S_ID, S_PARENT})
            set_scalar_kernel<<<(nw + 255) / 256, 256, 0, to->stream>>>(to->rec[to->cur], nw, s.rec,
                                                                         s.o_scal + slot, 0.0);
        CUDA_TRY(to, cudaGetLastError());
        CUDA_TRY(to, cudaStreamSynchronize(to->stream));
        to->nw = nw;
        to->next_id = 1.0;
        return ALEA_OK;
    }
    // positions: the source's rows, then a full evaluation in the destination
    CUDA_TRY(to, cudaSetDevice(from->device));
    const int n = from->sys.np * from->sys.dim;
    const long tot = static_cast<long>(n) * used;
    ++from->launches;
    to_rows_kernel<<<static_cast<int>((tot + 255) / 256), 256, 0, from->stream>>>(
        from->rec[from->cur], used, from->sys.rec, from->sys.o_pos, n, from->d_buf);
    CUDA_TRY(to, cudaGetLastError());
    CUDA_TRY(to, cudaStreamSynchronize(from->stream));
    CUDA_TRY(to, cudaSetDevice(to->device));
    const double* rows = from->d_buf;
    if (peer) {
        CUDA_TRY(to, cudaMemcpyPeerAsync(to->d_buf, to->device, from->d_buf, from->device,
                                         static_cast<size_t>(tot) * 8, to->stream));
        rows = to->d_buf;
    }
    return fresh_walkers(to, rows, used, nw);
}

// ───────────────────────── estimators ─────────────────────────────────

int alea_gpu_add_estimator(alea_gpu_ctx* c, const alea_gpu_estimator_spec* spec, int* id) {
    if (!c || !spec || !id) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_add_estimator: two-dimensional systems only");
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::string err;
    if (int rc = est_add(c->est, c->sys, *spec, c->stream, err, id)) return fail(c, rc, err);
    return ALEA_OK;
}

int alea_gpu_clear_estimators(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    est_free(c->est, c->stream);
    return ALEA_OK;
}

int alea_gpu_estimators_reset(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::string err;
    if (int rc = est_reset(c->est, c->stream, err)) return fail(c, rc, err);
    return ALEA_OK;
}

int alea_gpu_estimators_start_block(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::string err;
    if (int rc = est_start_block(c->est, c->stream, err)) return fail(c, rc, err);
    return ALEA_OK;
}

namespace {

// One measurement of the context's estimators: weights on the host (copied
// into the staging buffer), or the records' own (null), or all 1 (unit).
int measure_estimators(alea_gpu_ctx* c, const double* weights, bool unit, int chains) {
    if (est_count(c->est) == 0) return ALEA_OK;
    const double* dw = nullptr;
    if (weights && !unit) {
        CUDA_TRY(c, copy_in(c, c->d_buf, weights, sizeof(double) * c->nw));
        dw = c->d_buf;
    }
    std::string err;
    const EstSource src{records(c), c->sys.rec, c->sys.o_pos, c->sys.o_scal + S_WEIGHT, nullptr, c->nw};
    if (int rc = est_accumulate(c->est, c->sys, src, dw, unit, chains, c->pairs, c->npair, c->stream, err,
                                &c->launches))
        return fail(c, rc, err);
    return ALEA_OK;
}

int close_estimator_block(alea_gpu_ctx* c) {
    if (est_count(c->est) == 0) return ALEA_OK;
    std::string err;
    if (int rc = est_stop_block(c->est, c->stream, err, &c->d2h)) return fail(c, rc, err);
    return ALEA_OK;
}

}  // namespace

int alea_gpu_estimators_accumulate(alea_gpu_ctx* c, const double* weights, int n_chains) {
    const Phase phase("alea.estimators");
    if (!c) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    if (c->nw == 0) return fail(c, ALEA_ERR_INVALID, "no walkers");
    return measure_estimators(c, weights, false, n_chains);
}

int alea_gpu_estimators_stop_block(alea_gpu_ctx* c) {
    if (!c) return ALEA_ERR_INVALID;
    CUDA_TRY(c, cudaSetDevice(c->device));
    return close_estimator_block(c);
}

int alea_gpu_estimator_info(const alea_gpu_ctx* c, int id, alea_gpu_estimator_desc* out) {
    if (!c) return ALEA_ERR_INVALID;
    return est_info(c->est, id, out);
}

int alea_gpu_estimator_blocks(const alea_gpu_ctx* c, int id, double* blocks) {
    if (!c) return ALEA_ERR_INVALID;
    return est_blocks(c->est, id, blocks);
}

int alea_gpu_estimator_kvectors(const alea_gpu_ctx* c, int id, int* n1, int* n2, double* kx, double* ky,
                                int* shell_of, double* shell_k, int* shell_count) {
    if (!c) return ALEA_ERR_INVALID;
    return est_kvectors(c->est, id, n1, n2, kx, ky, shell_of, shell_k, shell_count);
}

// ───────────────────────── parameter derivatives ───────────────────────

namespace {

constexpr int kOrbitalGrid = 148 * 4;   // CTAs of the Gaussian-width kernel (walkers grid-strided)

int orbital_param_derivatives(alea_gpu_ctx* c, double* out, double* dgrad, double* dlap) {
    if (c->orbital_opts == 0) return ALEA_OK;
    const int grid = std::min(c->nw, kOrbitalGrid);
    if (!c->d_opt_scratch) {
        const size_t b = static_cast<size_t>(kOrbitalGrid) * 3 * c->sys.maxN * c->sys.maxN * 8;
        if (cudaMallocAsync(&c->d_opt_scratch, b, c->stream) != cudaSuccess)
            return fail(c, ALEA_ERR_NOMEM, "parameter derivatives: device allocation failed");
    }
    ++c->launches;
    CUDA_TRY(c, launch_orbital_param_derivatives(c->nw, grid, c->stream, c->sys, records(c), c->d_opt,
                                                 static_cast<int>(c->h_opt.size()), out, dgrad, dlap,
                                                 c->d_opt_scratch));
    return ALEA_OK;
}

}  // namespace

int alea_gpu_parameter_derivatives(alea_gpu_ctx* c, double* derivs, int* n_params) {
    const Phase phase("alea.param_derivs");
    if (!c || !n_params) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_parameter_derivatives: two-dimensional systems only");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const int nopt = static_cast<int>(c->h_opt.size());
    *n_params = nopt;
    if (!derivs || nopt == 0 || c->nw == 0) return ALEA_OK;
    if (c->sys.np > 256) return fail(c, ALEA_ERR_UNSUPPORTED, "parameter derivatives: more than 256 particles");
    if (!c->d_opt_out) {
        const size_t b = static_cast<size_t>(nopt) * c->capacity * 8;
        if (cudaMallocAsync(&c->d_opt_out, b, c->stream) != cudaSuccess)
            return fail(c, ALEA_ERR_NOMEM, "parameter derivatives: device allocation failed");
    }
    ++c->launches;
    CUDA_TRY(c, launch_param_derivatives(c->nw, c->stream, c->sys, records(c), c->d_opt, nopt, c->d_opt_out));
    if (int rc = orbital_param_derivatives(c, c->d_opt_out, nullptr, nullptr)) return rc;
    CUDA_TRY(c, copy_out(c, derivs, c->d_opt_out, static_cast<size_t>(nopt) * c->nw * 8));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

int alea_gpu_parameter_gradient_derivatives(alea_gpu_ctx* c, double* dgrad, double* dlap, int* n_params) {
    if (!c || !n_params) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_parameter_gradient_derivatives: two-dimensional systems only");
    CUDA_TRY(c, cudaSetDevice(c->device));
    const int nopt = static_cast<int>(c->h_opt.size());
    *n_params = nopt;
    if ((!dgrad && !dlap) || nopt == 0 || c->nw == 0) return ALEA_OK;
    bool backflow = false;
    for (const DevOpt& o : c->h_opt)
        if (o.kind == 2) {
            backflow = true;
            // η'' jumps at L when C = 2: the reference reports no curvature term there
            if (c->sys.bf[o.term].ch[o.ch].C < 3)
                return fail(c, ALEA_ERR_UNSUPPORTED, "curvature terms of a backflow channel with truncation C < 3");
        }
    if (c->sys.np > 256) return fail(c, ALEA_ERR_UNSUPPORTED, "parameter derivatives: more than 256 particles");
    if (backflow && bf_curvature_smem(c->sys) > 227 * 1024)
        return fail(c, ALEA_ERR_UNSUPPORTED, "backflow curvature terms: the block needs more than 227 KB of shared memory");
    const size_t cap = static_cast<size_t>(nopt) * c->sys.np * 2 * c->capacity;
    if (!c->d_opt_grad && cudaMallocAsync(&c->d_opt_grad, 2 * cap * 8, c->stream) != cudaSuccess)
        return fail(c, ALEA_ERR_NOMEM, "parameter derivatives: device allocation failed");
    const size_t n = static_cast<size_t>(nopt) * c->sys.np * 2 * c->nw;
    double* g = c->d_opt_grad;
    double* l = c->d_opt_grad + cap;
    CUDA_TRY(c, cudaMemsetAsync(g, 0, n * 8, c->stream));
    CUDA_TRY(c, cudaMemsetAsync(l, 0, n * 8, c->stream));
    ++c->launches;
    CUDA_TRY(c, launch_param_grad_derivatives(c->nw, c->stream, c->sys, records(c), c->d_opt, nopt, g, l));
    if (backflow) {
        ++c->launches;
        CUDA_TRY(c, launch_bf_curvature(c->nw, c->stream, c->sys, records(c), c->d_opt, nopt, g, l));
    }
    if (int rc = orbital_param_derivatives(c, nullptr, g, l)) return rc;
    if (dgrad) CUDA_TRY(c, copy_out(c, dgrad, g, n * 8));
    if (dlap) CUDA_TRY(c, copy_out(c, dlap, l, n * 8));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return ALEA_OK;
}

// ───────────────────────── forward walking API ─────────────────────────

int alea_gpu_set_forward_walking(alea_gpu_ctx* c, const double* lags, int n_lags, int interval) {
    if (!c || n_lags < 0 || (n_lags > 0 && !lags)) return ALEA_ERR_INVALID;
    if (c->sys.dim != 2) return fail(c, ALEA_ERR_UNSUPPORTED, "alea_gpu_set_forward_walking: two-dimensional systems only");
    CUDA_TRY(c, cudaSetDevice(c->device));
    fw_free(c);
    if (n_lags == 0) return ALEA_OK;
    if (interval < 1) return fail(c, ALEA_ERR_INVALID, "forward walking interval must be at least one step");
    for (int i = 0; i < n_lags; ++i) {
        if (!(std::isfinite(lags[i]) && lags[i] >= 0.0))
            return fail(c, ALEA_ERR_INVALID, "dmc: forward_walking lags must be finite and >= 0");
        if (i > 0 && !(lags[i] > lags[i - 1]))
            return fail(c, ALEA_ERR_INVALID, "dmc: forward_walking lags must be strictly increasing");
    }
    c->fw = new FwState();
    c->fw->lags.assign(lags, lags + n_lags);
    c->fw->interval = interval;
    c->fw->est.assign(static_cast<size_t>(n_lags), nullptr);
    return ALEA_OK;
}

int alea_gpu_add_fw_estimator(alea_gpu_ctx* c, int lag, const alea_gpu_estimator_spec* spec, int* id) {
    if (!c || !spec || !id) return ALEA_ERR_INVALID;
    if (!c->fw || lag < 0 || lag >= static_cast<int>(c->fw->lags.size()))
        return fail(c, ALEA_ERR_INVALID, "forward walking: no such lag (alea_gpu_set_forward_walking)");
    CUDA_TRY(c, cudaSetDevice(c->device));
    std::string err;
    if (int rc = est_add(c->fw->est[lag], c->sys, *spec, c->stream, err, id)) return fail(c, rc, err);
    return ALEA_OK;
}

int alea_gpu_fw_result(const alea_gpu_ctx* c, int lag, alea_gpu_fw_summary* out, double* block_potentials) {
    if (!c || !out || !c->fw || lag < 0 || lag >= static_cast<int>(c->fw->lags.size())) return ALEA_ERR_INVALID;
    const FwState* f = c->fw;
    *out = alea_gpu_fw_summary{};
    out->lag_time = f->lags[lag];
    if (f->lag_steps.size() != f->lags.size()) return ALEA_OK;   // no run yet
    out->lag_steps = static_cast<int>(f->lag_steps[lag]);
    out->measurements = f->measurements[lag];
    out->surviving_fraction =
        f->measurements[lag] > 0 ? f->surviving[lag] / static_cast<double>(f->measurements[lag]) : 0.0;
    const std::vector<double>& chain = f->block_pot[lag];
    out->n_blocks = static_cast<int>(chain.size());
    if (!chain.empty()) reblock(chain, out->potential, out->potential_error);
    if (block_potentials) std::copy(chain.begin(), chain.end(), block_potentials);
    return ALEA_OK;
}

int alea_gpu_fw_estimator_info(const alea_gpu_ctx* c, int lag, int id, alea_gpu_estimator_desc* out) {
    if (!c || !c->fw || lag < 0 || lag >= static_cast<int>(c->fw->lags.size())) return ALEA_ERR_INVALID;
    return est_info(c->fw->est[lag], id, out);
}

int alea_gpu_fw_estimator_blocks(const alea_gpu_ctx* c, int lag, int id, double* blocks) {
    if (!c || !c->fw || lag < 0 || lag >= static_cast<int>(c->fw->lags.size())) return ALEA_ERR_INVALID;
    return est_blocks(c->fw->est[lag], id, blocks);
}

int alea_gpu_fw_estimator_kvectors(const alea_gpu_ctx* c, int lag, int id, int* n1, int* n2, double* kx,
                                   double* ky, int* shell_of, double* shell_k, int* shell_count) {
    if (!c || !c->fw || lag < 0 || lag >= static_cast<int>(c->fw->lags.size())) return ALEA_ERR_INVALID;
    return est_kvectors(c->fw->est[lag], id, n1, n2, kx, ky, shell_of, shell_k, shell_count);
}

int alea_gpu_vmc_run(alea_gpu_ctx* c, const alea_gpu_run_config* cfg, alea_gpu_run_result* res,
                     double* block_energies) {
    const Phase phase("alea.vmc_run");
    if (!c || !cfg || !res) return ALEA_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    const int nw = c->nw;
    const int T = std::min(std::max(cfg->n_streams, 1), nw);
    if (int rc = alea_gpu_set_streams(c, cfg->seed, ALEA_STREAM_VMC, T)) return rc;
    alea_gpu_vmc_params prm{cfg->tau, cfg->n_substeps, cfg->use_drift};
    std::vector<double> blocks;   // [T][n_acc], chain-major
    std::vector<std::vector<double>> chain(T);
    double e_sum = 0, e2_sum = 0;
    int64_t n_tot = 0, acc = 0, prop = 0, all_moves = 0, all_evals = 0;
    const int base = nw / T, rem = nw % T;
    std::string est_err;
    if (int rc = est_reset(c->est, c->stream, est_err)) return fail(c, rc, est_err);
    for (int b = 0; b < cfg->n_equilibration_blocks + cfg->n_accumulation_blocks; ++b) {
        const bool measure = b >= cfg->n_equilibration_blocks;
        if (measure)
            if (int rc = est_start_block(c->est, c->stream, est_err)) return fail(c, rc, est_err);
        std::vector<double> blk(T, 0.0);
        std::vector<int64_t> blk_n(T, 0);
        for (int st = 0; st < cfg->n_steps; ++st) {
            if (c->cancel && c->cancel->load(std::memory_order_relaxed))
                return fail(c, ALEA_ERR_CANCELLED, "cancelled");
            alea_gpu_step_stats s{};
            if (int rc = alea_gpu_vmc_step(c, &prm, &s)) return rc;
            all_moves += s.n_proposed;
            all_evals += s.n_walkers;
            if (!measure) continue;
            if (int rc = measure_estimators(c, nullptr, true, T)) return rc;
            std::vector<double> el;
            if (int rc = read_scalars(c, S_EL, el)) return rc;
            for (int t = 0; t < T; ++t) {
                const int w0 = t * base + std::min(t, rem), cnt = base + (t < rem ? 1 : 0);
                for (int w = w0; w < w0 + cnt; ++w) {
                    blk[t] += el[w];
                    e_sum += el[w];
                    e2_sum += el[w] * el[w];
                }
                blk_n[t] += cnt;
                n_tot += cnt;
            }
            acc += s.n_accepted;
            prop += s.n_proposed;
        }
        if (measure) {
            for (int t = 0; t < T; ++t) chain[t].push_back(blk[t] / static_cast<double>(blk_n[t]));
            if (int rc = close_estimator_block(c)) return rc;
        }
    }
    for (int t = 0; t < T; ++t) blocks.insert(blocks.end(), chain[t].begin(), chain[t].end());
    double mean = 0.0, err = 0.0;
    reblock(blocks, mean, err);
    res->energy = mean;
    res->energy_error = err;
    const double m = n_tot ? e_sum / static_cast<double>(n_tot) : 0.0;
    res->variance = n_tot ? e2_sum / static_cast<double>(n_tot) - m * m : 0.0;
    res->acceptance = prop ? static_cast<double>(acc) / static_cast<double>(prop) : 0.0;
    res->walltime_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->n_walkers = c->nw;
    res->e_trial = 0.0;
    res->n_moves = all_moves;
    res->n_evaluations = all_evals;
    if (block_energies) std::copy(blocks.begin(), blocks.end(), block_energies);
    return ALEA_OK;
}

int alea_gpu_dmc_run(alea_gpu_ctx* c, const alea_gpu_run_config* cfg, alea_gpu_run_result* res,
                     double* block_energies) {
    const Phase phase("alea.dmc_run");
    if (!c || !cfg || !res) return ALEA_ERR_INVALID;
    const auto t0 = std::chrono::steady_clock::now();
    const int target = cfg->target_walkers > 0 ? cfg->target_walkers : c->nw;
    const int n_threads = std::max(1, std::min(cfg->n_streams > 0 ? cfg->n_streams : c->nw, c->nw));
    if (int rc = alea_gpu_set_streams(c, cfg->seed, ALEA_STREAM_DMC, n_threads)) return rc;
    HostXo brng(stream_seed(cfg->seed, ALEA_STREAM_BRANCH, 0));
    uint64_t bstate[4];
    std::memcpy(bstate, brng.s, 32);
    // diffusing particles (dmc.cpp:50-66)
    double max_inv = 0.0;
    for (double x : c->h_inv_mass) max_inv = std::max(max_inv, x);
    int n_diff = 0;
    for (int g = 0; g < c->sys.ngroups; ++g) {
        const int i = c->sys.gfirst[g];
        const double gi = std::max(c->h_inv_mass[i * 2], c->h_inv_mass[i * 2 + 1]);
        if (gi >= 1e-3 * max_inv) n_diff += c->sys.glast[g] - c->sys.gfirst[g];
    }
    n_diff = std::max(n_diff, 1);
    const double tau = cfg->tau;
    const double t_step = tau * std::max(1, cfg->n_substeps);
    const double feedback = (t_step > 0.0 && cfg->population_generations > 0.0)
                                ? 1.0 / (cfg->population_generations * t_step) : 0.0;
    const double alpha = cfg->branch_cutoff_alpha > 0.0 ? cfg->branch_cutoff_alpha : 2.0;
    std::vector<double> el;
    if (int rc = read_scalars(c, S_EL, el)) return rc;
    double e0 = 0.0;
    for (double x : el) e0 += x;
    double etrial = e0 / static_cast<double>(c->nw), eref = etrial, eref_sum = 0.0, eref_wsum = 0.0;
    double e_cut = INFINITY, e_max = INFINITY;
    auto refresh_spread = [&](const std::vector<double>& e) {
        const double sigma = robust_spread(e.data(), e.size());
        if (!(std::isfinite(sigma) && sigma > 0.0 && tau > 0.0)) {
            e_cut = e_max = INFINITY;
        } else {
            e_cut = alpha * std::sqrt(sigma * std::sqrt(static_cast<double>(n_diff)) / tau);
            e_max = 1.5 * e_cut;
        }
    };
    refresh_spread(el);
    std::vector<double> blocks;
    int64_t acc = 0, prop = 0, all_evals = 0;
    std::string est_err;
    if (int rc = est_reset(c->est, c->stream, est_err)) return fail(c, rc, est_err);
    if (int rc = fw_prepare(c, cfg)) return rc;
    long step_index = 0;   // from the first equilibration step (forward walking's clock)
    for (int b = 0; b < cfg->n_equilibration_blocks + cfg->n_accumulation_blocks; ++b) {
        const bool measure = b >= cfg->n_equilibration_blocks;
        if (b == cfg->n_equilibration_blocks) {
            eref_sum = eref_wsum = 0.0;
            // milestone: the equilibrated population (dmc.cpp:776-779)
            if (c->ckpt_fn) c->ckpt_fn(c->ckpt_user, c, "eq", 0);
        }
        if (measure) {
            if (int rc = est_start_block(c->est, c->stream, est_err)) return fail(c, rc, est_err);
            if (int rc = fw_start_block(c)) return rc;
        }
        double blk_e = 0.0, blk_w = 0.0;
        for (int st = 0; st < cfg->n_steps; ++st) {
            if (c->cancel && c->cancel->load(std::memory_order_relaxed))
                return fail(c, ALEA_ERR_CANCELLED, "cancelled");
            alea_gpu_dmc_params prm{tau, cfg->n_substeps, etrial, eref, e_cut, e_max};
            alea_gpu_step_stats s{};
            if (int rc = alea_gpu_dmc_advance(c, &prm, &s)) return rc;
            acc += s.n_accepted;
            prop += s.n_proposed;
            all_evals += static_cast<int64_t>(std::max(1, cfg->n_substeps)) * s.n_walkers;
            blk_e += s.energy_sum;
            blk_w += s.weight_sum;
            const double ens_e = s.weight_sum > 0.0 ? s.energy_sum / s.weight_sum : etrial;
            // mixed estimator: the population before the branch, DMC weights
            if (measure)
                if (int rc = measure_estimators(c, nullptr, false, 1)) return rc;
            // pure estimators: snapshots and lagged measurements, same weights
            if (int rc = fw_observe(c, step_index)) return rc;
            if (int rc = alea_gpu_dmc_branch(c, bstate, target)) return rc;
            fw_branch(c);
            ++step_index;
            if (measure) {
                eref_sum += ens_e * s.weight_sum;
                eref_wsum += s.weight_sum;
                if (eref_wsum > 0.0) eref = eref_sum / eref_wsum;
            } else {
                eref = ens_e;
            }
            if (s.weight_sum > 0.0)
                etrial = eref - feedback * std::log(s.weight_sum / static_cast<double>(target));
        }
        if (measure) {
            blocks.push_back(blk_w > 0.0 ? blk_e / blk_w : 0.0);
            if (int rc = close_estimator_block(c)) return rc;
            if (int rc = fw_stop_block(c)) return rc;
            // quarter milestones (dmc.cpp:810-821): integer quarters, each once
            if (c->ckpt_fn) {
                const int n_acc = cfg->n_accumulation_blocks, done = b - cfg->n_equilibration_blocks + 1;
                if (done == n_acc / 4)
                    c->ckpt_fn(c->ckpt_user, c, "a25", done);
                else if (done == n_acc / 2 && n_acc / 2 > n_acc / 4)
                    c->ckpt_fn(c->ckpt_user, c, "a50", done);
                else if (done == 3 * n_acc / 4 && 3 * n_acc / 4 > n_acc / 2)
                    c->ckpt_fn(c->ckpt_user, c, "a75", done);
            }
        } else {
            if (int rc = read_scalars(c, S_EL, el)) return rc;
            refresh_spread(el);
        }
    }
    double mean = 0.0, err = 0.0;
    reblock(blocks, mean, err);
    res->energy = mean;
    res->energy_error = err;
    double var = 0.0;
    for (double x : blocks) var += (x - mean) * (x - mean);
    res->variance = blocks.size() >= 2 ? var / static_cast<double>(blocks.size() - 1) : 0.0;
    res->acceptance = prop ? static_cast<double>(acc) / static_cast<double>(prop) : 0.0;
    res->walltime_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    res->n_walkers = c->nw;
    res->e_trial = etrial;
    res->n_moves = prop;
    res->n_evaluations = all_evals;
    if (block_energies) std::copy(blocks.begin(), blocks.end(), block_energies);
    return ALEA_OK;
}

}  // extern "C"

// ───────────────────────── internal: serving support ───────────────────

namespace alea_gpu {

void set_cancel_flag(alea_gpu_ctx* c, const std::atomic<int>* flag) {
    if (c) c->cancel = flag;
}

// Device bytes a context of `capacity` walkers of `sys` will hold, from the
// record layout of build_system (hot part, orbital rows, image sums), both
// record buffers, staging, one sweep's randoms per substep and the pair list.
size_t footprint_bytes(const alea_gpu_system* sys, int capacity, int n_substeps) {
    if (!sys || capacity < 1) return 0;
    const long np = sys->n_particles;
    if (sys->dim == 3) {   // build_system3's record: 7 planes of 3N, scalars, per determinant x, A, F, (ln|det|, sign)
        long rec = 21 * np + S_NSCAL;
        const int ndet = sys->n_backflow > 0 ? sys->n_backflow : sys->n_blocks;
        for (int d = 0; d < ndet; ++d) {
            const long n = sys->n_backflow > 0 ? sys->backflow[d].last - sys->backflow[d].first
                                               : sys->blocks[d].last - sys->blocks[d].first;
            rec += 2 * round4(3 * n) + round4(n * n) + 4;
        }
        rec = round4(rec);
        const size_t cap = static_cast<size_t>(capacity);
        size_t bytes = 2 * cap * static_cast<size_t>(rec) * 8;
        bytes += cap * static_cast<size_t>(std::max<long>(3 * np, 8)) * 8 + cap * 5;
        bytes += static_cast<size_t>(std::max(n_substeps, 1)) * static_cast<size_t>(np) * 4 * cap * 8;
        bytes += static_cast<size_t>(np) * static_cast<size_t>(np) * 4 + (1u << 20);
        return bytes;
    }
    bool cplx = false;
    for (int b = 0; b < sys->n_blocks; ++b) cplx |= sys->blocks[b].type == ALEA_ORB_TWISTED_PLANE_WAVE;
    long rec = 14 * np + S_NSCAL + (cplx ? 4 * np : 0);
    for (int b = 0; b < sys->n_blocks; ++b) {
        const long n = sys->blocks[b].last - sys->blocks[b].first;
        rec += (cplx ? 2 : 1) * round4(n * n) + round4(n);
        if (!cplx) rec += round4(n * n) + 2 * round4(2 * n * n);
    }
    for (int d = 0; d < sys->n_backflow; ++d) {
        const long n = sys->backflow[d].last - sys->backflow[d].first;
        rec += round4(2 * n) + round4(n * n) + round4(2 * n) + 4;
    }
    long nk = 0;
    for (int t = 0; t < sys->n_terms; ++t) nk = std::max<long>(nk, sys->terms[t].kset.n_k);
    rec += 2L * sys->n_groups * nk;
    rec = round4(rec);
    const size_t cap = static_cast<size_t>(capacity);
    size_t bytes = 2 * cap * static_cast<size_t>(rec) * 8;
    bytes += cap * static_cast<size_t>(std::max<long>(2 * np, 8)) * 8 + cap * 5;
    bytes += static_cast<size_t>(std::max(n_substeps, 1)) * static_cast<size_t>(np) * 3 * cap * 8;
    bytes += static_cast<size_t>(np) * static_cast<size_t>(np) * 4 + (1u << 20);
    return bytes;
}

}  // namespace alea_gpu
