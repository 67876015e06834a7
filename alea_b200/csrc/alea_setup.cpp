// Host-side system setup: the tables the walker kernels read, computed once
// before a run (the device never fits anything).  The equivalent of the
// reference's builders for the systems this library runs:
//
//   cell             lattice from r_s and N (src/qmc/app.cpp:288-336)
//   plane waves      closed reciprocal shells (src/wavefunction/orbital_set.h:575-665)
//   cusps            Kato Γ = 2 μ R / (2ℓ + d − 1) (src/builders/jastrow.cpp:48-98)
//   Ewald            optimized breakup of 1/r (alea_breakup.cpp; the reference's
//                    src/numerics/ewald_breakup.cpp:205-276 fits the same χ²)
//   Padé image sum   u − u∞ split by the same breakup with the Jastrow options
//                    (src/wavefunction/periodic_pair_sum.cpp:21-60)
//   initial walkers  App::initialize_positions (src/qmc/app.cpp:56-112)
#include <algorithm>
#include <array>
#include <mutex>
#include <map>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <limits>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/alea_gpu.h"
#include "alea_breakup.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 2.0 * kPi;

// ───────────────────────── cell, shells ─────────────────────────────────

struct Cell {
    double a[4] = {0, 0, 0, 0};   // reduced rows
    double b[4] = {0, 0, 0, 0};   // reciprocal, b_i · a_j = 2π δ_ij
    double area = 0.0, ws = 0.0;
};

// Lattice rows a = (a1, a2) as the device context reduces them: rows along
// the axes are permuted onto x, y; any other pair is Lagrange-Gauss reduced.
// Reciprocal vectors and k indices then refer to the same basis as the
// device's ladders.
void reduce_lattice(double a[4]) {
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
        std::copy(r, r + 4, a);
        return;
    }
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

Cell make_cell(const double a_in[4]) {
    Cell c;
    std::copy(a_in, a_in + 4, c.a);
    reduce_lattice(c.a);
    const double det = c.a[0] * c.a[3] - c.a[1] * c.a[2];
    if (det == 0.0) throw std::invalid_argument("cell: singular lattice vectors");
    c.area = std::abs(det);
    const double inv = 1.0 / det;
    const double ainv[4] = {c.a[3] * inv, -c.a[2] * inv, -c.a[1] * inv, c.a[0] * inv};
    for (int k = 0; k < 4; ++k) c.b[k] = kTwoPi * ainv[k];
    double shortest2 = 0.0;
    for (int n0 = -2; n0 <= 2; ++n0)
        for (int n1 = -2; n1 <= 2; ++n1) {
            if (n0 == 0 && n1 == 0) continue;
            const double x = n0 * c.a[0] + n1 * c.a[2], y = n0 * c.a[1] + n1 * c.a[3];
            const double r2 = x * x + y * y;
            if (shortest2 == 0.0 || r2 < shortest2) shortest2 = r2;
        }
    c.ws = 0.5 * std::sqrt(shortest2);
    return c;
}

Cell make_cell(double lx, double ly) {
    const double a[4] = {lx, 0.0, 0.0, ly};
    return make_cell(a);
}

// ∫ outside the Wigner-Seitz cell of a radial function, as ∮ dθ f(ρ(θ)) with
// ρ(θ) = min over lattice translations L (u·L > 0) of |L|²/(2 u·L), by a
// 2^18-point midpoint rule in θ (its error comes only from the cell's
// corners, ~1e-10 relative).  f(ρ) = ∫_ρ^∞ v(r) r dr is the caller's tail.
template <class F>
double ws_exterior_integral(const Cell& c, F&& f) {
    std::vector<double> lx, ly;
    for (int s = -2; s <= 2; ++s)
        for (int t = -2; t <= 2; ++t) {
            if (s == 0 && t == 0) continue;
            lx.push_back(s * c.a[0] + t * c.a[2]);
            ly.push_back(s * c.a[1] + t * c.a[3]);
        }
    constexpr size_t n_theta = size_t{1} << 18;
    const double dtheta = kTwoPi / static_cast<double>(n_theta);
    double sum = 0.0;
    for (size_t k = 0; k < n_theta; ++k) {
        const double theta = (static_cast<double>(k) + 0.5) * dtheta;
        const double ux = std::cos(theta), uy = std::sin(theta);
        double rho = std::numeric_limits<double>::infinity();
        for (size_t q = 0; q < lx.size(); ++q) {
            const double proj = ux * lx[q] + uy * ly[q];
            if (proj > 0.0) rho = std::min(rho, 0.5 * (lx[q] * lx[q] + ly[q] * ly[q]) / proj);
        }
        sum += f(rho);
    }
    return sum * dtheta;
}

// The first `want` real plane waves of closed reciprocal shells (k = 0 gives
// one cosine, every ±k pair a cosine and a sine).
void plane_wave_shells(const Cell& c, int want, std::vector<double>& k, std::vector<int>& is_sin) {
    const double* b = c.b;
    const double area = std::abs(b[0] * b[3] - b[1] * b[2]);
    const double h_min = area / std::max(std::hypot(b[0], b[1]), std::hypot(b[2], b[3]));
    struct Kv { double k2, x, y; };
    std::vector<int> closed;
    for (int M = 4; M <= 4096; M *= 2) {
        const double r2 = (M * h_min) * (M * h_min) * (1.0 + 1e-12);
        std::vector<Kv> kv;
        for (int i = -M; i <= M; ++i)
            for (int j = -M; j <= M; ++j) {
                Kv e{0, i * b[0] + j * b[2], i * b[1] + j * b[3]};
                e.k2 = e.x * e.x + e.y * e.y;
                if (e.k2 <= r2) kv.push_back(e);
            }
        std::sort(kv.begin(), kv.end(), [](const Kv& p, const Kv& q) {
            if (p.k2 != q.k2) return p.k2 < q.k2;
            if (p.x != q.x) return p.x < q.x;
            return p.y < q.y;
        });
        k.clear();
        is_sin.clear();
        closed.clear();
        size_t s = 0;
        while (s < kv.size()) {
            size_t e = s + 1;
            while (e < kv.size() && std::abs(kv[e].k2 - kv[s].k2) <= 1e-9 * (1.0 + kv[s].k2)) ++e;
            if (kv[s].k2 <= 1e-12 * (1.0 + kv[s].k2)) {
                k.push_back(0.0);
                k.push_back(0.0);
                is_sin.push_back(0);
            } else {
                for (size_t q = s; q < e; ++q) {
                    const bool positive = kv[q].x > 1e-12 || (!(kv[q].x < -1e-12) && kv[q].y > 1e-12);
                    if (!positive) continue;
                    for (int which = 0; which < 2; ++which) {
                        k.push_back(kv[q].x);
                        k.push_back(kv[q].y);
                        is_sin.push_back(which);
                    }
                }
            }
            closed.push_back(static_cast<int>(is_sin.size()));
            s = e;
        }
        if (static_cast<int>(is_sin.size()) >= want) break;
    }
    if (std::find(closed.begin(), closed.end(), want) == closed.end())
        throw std::invalid_argument("plane waves: " + std::to_string(want) +
                                    " orbitals leave a reciprocal shell partly filled");
    k.resize(2 * static_cast<size_t>(want));
    is_sin.resize(want);
}

// The n lowest |k + θ| of the reciprocal lattice at twist θ = t_x b1 + t_y b2
// (TwistedPlaneWaveOrbitalSet's occupation, complex_orbital_set.h:278-343):
// enumerate the |i|, |j| <= M box, sort by |q|², grow M until every q with
// |q| <= M h_min - |θ| is in the box, and refuse a twist at which the n-th
// orbital splits a degenerate shell.  q holds (q_x, q_y) per orbital.
void twisted_shells(const Cell& c, int n, double tx, double ty, std::vector<double>& q) {
    const double* b = c.b;
    const double th[2] = {tx * b[0] + ty * b[2], tx * b[1] + ty * b[3]};
    const double th_norm = std::hypot(th[0], th[1]);
    const double area = std::abs(b[0] * b[3] - b[1] * b[2]);
    const double h_min = area / std::max(std::hypot(b[0], b[1]), std::hypot(b[2], b[3]));
    struct Q { double q2, x, y; };
    for (int M = 4; M <= 4096; M *= 2) {
        std::vector<Q> qs;
        for (int i = -M; i <= M; ++i)
            for (int j = -M; j <= M; ++j) {
                const double x = i * b[0] + j * b[2] + th[0];
                const double y = i * b[1] + j * b[3] + th[1];
                qs.push_back({x * x + y * y, x, y});
            }
        if (qs.size() <= static_cast<size_t>(n)) continue;
        std::stable_sort(qs.begin(), qs.end(), [](const Q& a, const Q& z) { return a.q2 < z.q2; });
        const double r_safe = M * h_min - th_norm;
        if (r_safe <= 0.0 || qs[n].q2 > r_safe * r_safe) continue;
        if (n > 0 && std::abs(qs[n].q2 - qs[n - 1].q2) <= 1e-9 * (1.0 + qs[n].q2))
            throw std::invalid_argument("twisted plane waves: " + std::to_string(n) +
                                        " orbitals split a degenerate |k+theta| shell at this twist");
        q.clear();
        for (int k = 0; k < n; ++k) {
            q.push_back(qs[k].x);
            q.push_back(qs[k].y);
        }
        return;
    }
    throw std::invalid_argument("twisted plane waves: enumeration did not converge");
}

// ───────────────────────── JSON ─────────────────────────────────────────

struct Json {
    std::string s;
    bool first = true;
    void sep() {
        if (!first) s += ",";
        first = false;
    }
    void key(const std::string& k) {
        sep();
        s += "\"" + k + "\":";
        first = true;
    }
    void num(double x) {
        sep();
        char b[40];
        std::snprintf(b, sizeof b, "%.17g", x);
        s += b;
    }
    void open(char c) {
        sep();
        s += c;
        first = true;
    }
    void close(char c) {
        s += c;
        first = false;
    }
    template <class V>
    void arr(const std::string& k, const V& v) {
        if (!k.empty()) key(k);
        open('[');
        for (auto x : v) num(static_cast<double>(x));
        close(']');
    }
    void kv(const std::string& k, double x) {
        key(k);
        num(x);
    }
    void ks(const std::string& k, const std::string& x) {
        key(k);
        sep();
        s += "\"" + x + "\"";
    }
};

}  // namespace

// ───────────────────────── setup object ─────────────────────────────────

struct alea_gpu_setup {
    alea_gpu_system sys{};
    std::string json;
    std::string err;
    // owned tables
    std::vector<std::vector<double>> dv;
    std::vector<std::vector<int>> iv;
    std::vector<double> anchors;   // [np*2] crystal sites (empty: uniform)
    double jitter = 0.0;
    double open_L = 1.0;
    const double* keep(std::vector<double> v) {
        dv.push_back(std::move(v));
        return dv.back().data();
    }
    const int* keepi(std::vector<int> v) {
        iv.push_back(std::move(v));
        return iv.back().data();
    }
};

namespace {

using Breakup = alea_breakup::Result;

void set_spline(alea_gpu_setup* S, alea_gpu_spline& sp, const Breakup& br) {
    sp.r_cut = br.rc;
    sp.inv_delta = 1.0 / br.delta;
    sp.n_knots = br.n_knots;
    sp.scaled = S->keep(br.scaled);
}
void set_kset(alea_gpu_setup* S, alea_gpu_kset& ks, const Breakup& br) {
    ks.n_k = static_cast<int>(br.weight.size());
    ks.n1 = S->keepi(br.n[0]);
    ks.n2 = S->keepi(br.n[1]);
    ks.kx = S->keep(br.kvec[0]);
    ks.ky = S->keep(br.kvec[1]);
    ks.weight = S->keep(br.weight);
}

alea_breakup::Lattice lattice_of(const Cell& c) {
    alea_breakup::Lattice lat;
    lat.dim = 2;
    std::copy(c.a, c.a + 4, lat.a);
    std::copy(c.b, c.b + 4, lat.b);
    lat.volume = c.area;
    return lat;
}

// Coulomb 1/(ε r) Ewald tables (n_knots auto-tuned, default k set).
// Breakups depend only on the cell and the radial function's parameters;
// builders of the same cell (twists of one electron gas, say) reuse them.
std::mutex g_breakup_mu;
std::map<std::vector<double>, Breakup> g_breakups;
std::map<std::vector<double>, double> g_breakup_uinf;

std::vector<double> breakup_key(const Cell& c, double kind, std::initializer_list<double> extra) {
    std::vector<double> key{kind, c.a[0], c.a[1], c.a[2], c.a[3]};
    key.insert(key.end(), extra.begin(), extra.end());
    return key;
}

// The knot count is the smallest of 12, 16, 20, 24 whose fit misfit on the
// lattice shells is below `tol`.  The fit targets leave out r < r_c 2⁻⁴⁷ as
// the reference's do (src/numerics/long_range_breakup.cpp fit_target), so
// that the tables, and the local energies to 1e-10, are the reference's.
Breakup ewald_breakup_uncached(const Cell& c, double tol) {
    const auto f = alea_breakup::coulomb(std::ldexp(1.0, -47));
    for (int nk : {12, 16, 20, 24}) {
        alea_breakup::Options opt;
        opt.n_knots = nk;
        Breakup br = alea_breakup::optimize(lattice_of(c), c.ws, *f, opt);
        if (br.residual < tol) return br;
    }
    throw std::runtime_error("ewald: the breakup did not reach the requested tolerance");
}

Breakup ewald_breakup(const Cell& c, double tol) {
    const std::vector<double> key = breakup_key(c, 0.0, {tol});
    {
        std::lock_guard<std::mutex> lk(g_breakup_mu);
        auto it = g_breakups.find(key);
        if (it != g_breakups.end()) return it->second;
    }
    Breakup br = ewald_breakup_uncached(c, tol);
    std::lock_guard<std::mutex> lk(g_breakup_mu);
    g_breakups[key] = br;
    return br;
}

// Image-summed Padé tables (the Jastrow breakup options).
Breakup pade_breakup(const Cell& c, const std::vector<double>& a, const std::vector<double>& b,
                     double& u_inf) {
    std::vector<double> key = breakup_key(c, 1.0, {static_cast<double>(a.size())});
    key.insert(key.end(), a.begin(), a.end());
    key.insert(key.end(), b.begin(), b.end());
    {
        std::lock_guard<std::mutex> lk(g_breakup_mu);
        auto it = g_breakups.find(key);
        if (it != g_breakups.end()) {
            u_inf = g_breakup_uinf[key];
            return it->second;
        }
    }
    const auto f = alea_breakup::rational(a, b, &u_inf);
    // the Jastrow's options: a shorter continuum and k_cut = 5 |b|_min
    alea_breakup::Options opt;
    opt.k_continuum = 20.0 * kPi / c.ws;
    opt.k_max = 300.0 / c.ws;
    opt.n_continuum = 150;
    opt.k_cut = 5.0 * std::min(std::hypot(c.b[0], c.b[1]), std::hypot(c.b[2], c.b[3]));
    Breakup br = alea_breakup::optimize(lattice_of(c), c.ws, *f, opt);
    std::lock_guard<std::mutex> lk(g_breakup_mu);
    g_breakups[key] = br;
    g_breakup_uinf[key] = u_inf;
    return br;
}

void json_spline(Json& j, const std::string& k, const alea_gpu_spline& sp) {
    j.key(k);
    j.open('{');
    j.kv("r_cut", sp.r_cut);
    j.kv("inv_delta", sp.inv_delta);
    j.kv("n_knots", sp.n_knots);
    j.arr("scaled", std::vector<double>(sp.scaled, sp.scaled + 3 * sp.n_knots));
    j.close('}');
}
void json_kset(Json& j, const alea_gpu_kset& ks) {
    j.arr("n1", std::vector<int>(ks.n1, ks.n1 + ks.n_k));
    j.arr("n2", std::vector<int>(ks.n2, ks.n2 + ks.n_k));
    j.arr("kx", std::vector<double>(ks.kx, ks.kx + ks.n_k));
    j.arr("ky", std::vector<double>(ks.ky, ks.ky + ks.n_k));
    j.arr("weight", std::vector<double>(ks.weight, ks.weight + ks.n_k));
}

// The system description as JSON (the schema alea_b200.pack_system reads).
void write_json(alea_gpu_setup* S, const std::string& kind, double ewald_self, double ewald_bg) {
    const alea_gpu_system& y = S->sys;
    Json j;
    j.open('{');
    j.ks("kind", kind);
    j.kv("dim", y.dim);
    j.kv("np", y.n_particles);
    j.key("cell");
    j.open('{');
    j.kv("periodic", y.periodic);
    j.kv("dim", y.dim);
    if (y.periodic) j.arr("vectors", std::vector<double>(y.lattice, y.lattice + 4));
    j.close('}');
    j.key("groups");
    j.open('[');
    for (int g = 0; g < y.n_groups; ++g) {
        j.open('{');
        j.kv("first", y.groups[g].first);
        j.kv("last", y.groups[g].last);
        j.kv("charge", y.groups[g].charge);
        j.arr("inv_mass", std::vector<double>(y.groups[g].inv_mass, y.groups[g].inv_mass + 2));
        j.close('}');
    }
    j.close(']');
    j.key("slater");
    j.open('[');
    for (int b = 0; b < y.n_blocks; ++b) {
        const alea_gpu_orbitals& B = y.blocks[b];
        const int n = B.last - B.first;
        j.open('{');
        j.kv("first", B.first);
        j.kv("last", B.last);
        if (B.type == ALEA_ORB_PLANE_WAVE) {
            j.ks("type", "plane_wave");
            j.arr("k", std::vector<double>(B.k, B.k + 2 * n));
            j.arr("is_sin", std::vector<int>(B.is_sin, B.is_sin + n));
        } else if (B.type == ALEA_ORB_TWISTED_PLANE_WAVE) {
            j.ks("type", "twisted_plane_wave");
            j.arr("q", std::vector<double>(B.k, B.k + 2 * n));
        } else {
            j.ks("type", "gaussian");
            j.arr("centers", std::vector<double>(B.centers, B.centers + 2 * n));
            j.arr("alphas", std::vector<double>(B.alphas, B.alphas + n));
        }
        j.close('}');
    }
    j.close(']');
    j.key("pade");
    j.open('[');
    for (int t = 0; t < y.n_terms; ++t) {
        const alea_gpu_pair_term& T = y.terms[t];
        if (T.kind != ALEA_PAIR_PADE) continue;
        j.open('{');
        j.arr("ga", std::vector<int>{T.pairs[0][0], T.pairs[0][1]});
        j.arr("gb", std::vector<int>{T.pairs[0][2], T.pairs[0][3]});
        j.arr("a", std::vector<double>(T.coeffs, T.coeffs + T.num_order));
        j.arr("b", std::vector<double>(T.coeffs + T.num_order, T.coeffs + T.num_order + T.den_order));
        if (T.image_sum) {
            j.key("image_sum");
            j.open('{');
            json_spline(j, "spline", T.short_range);
            j.kv("u_inf", T.u_inf);
            json_kset(j, T.kset);
            j.close('}');
        }
        if (T.n_opt > 0) {
            j.key("opt");
            j.open('[');
            for (int q = 0; q < T.n_opt; ++q) {
                j.open('{');
                j.kv("index", T.opt_index[q]);
                if (T.image_sum) {
                    j.kv("inf", T.opt_inf[q]);
                    json_spline(j, "spline", T.opt_short_range[q]);
                    j.arr("weight", std::vector<double>(T.opt_weight[q], T.opt_weight[q] + T.kset.n_k));
                }
                j.close('}');
            }
            j.close(']');
        }
        j.close('}');
    }
    j.close(']');
    j.key("drummond");
    j.open('[');
    for (int t = 0; t < y.n_terms; ++t) {
        const alea_gpu_pair_term& T = y.terms[t];
        if (T.kind != ALEA_PAIR_DRUMMOND) continue;
        j.open('{');
        j.kv("C", T.C);
        j.kv("gamma", T.gamma);
        j.kv("L", T.L);
        j.arr("coeffs", std::vector<double>(T.dcoeffs, T.dcoeffs + T.n_coeffs));
        j.key("pairs");
        j.open('[');
        for (int q = 0; q < T.n_pairs; ++q)
            j.arr("", std::vector<int>{T.pairs[q][0], T.pairs[q][1], T.pairs[q][2], T.pairs[q][3]});
        j.close(']');
        j.close('}');
    }
    j.close(']');
    if (y.ewald.enabled) {
        j.key("ewald");
        j.open('{');
        j.kv("r_cut", y.ewald.r_cut);
        json_spline(j, "spline", y.ewald.long_range);
        json_kset(j, y.ewald.kset);
        j.kv("inv_eps", y.ewald.inv_eps);
        j.kv("self_energy", ewald_self);
        j.kv("background_energy", ewald_bg);
        j.close('}');
    }
    j.key("coulomb");
    j.open('[');
    for (int cidx = 0; cidx < y.n_coulomb; ++cidx) {
        const alea_gpu_coulomb& C = y.coulomb[cidx];
        j.open('{');
        j.arr("ga", std::vector<int>{C.a_first, C.a_last});
        j.arr("gb", std::vector<int>{C.b_first, C.b_last});
        j.kv("coef", C.coef);
        j.close('}');
    }
    j.close(']');
    j.key("zero_energy");
    j.open('[');
    for (int t = 0; t < y.n_terms; ++t) {
        const alea_gpu_pair_term& T = y.terms[t];
        if (T.kind != ALEA_PAIR_ZERO_ENERGY) continue;
        j.open('{');
        j.arr("ga", std::vector<int>{T.pairs[0][0], T.pairs[0][1]});
        j.arr("gb", std::vector<int>{T.pairs[0][2], T.pairs[0][3]});
        j.kv("b", T.ze_b);
        j.kv("exponent", T.ze_exponent);
        j.kv("matching_radius", T.ze_matching_radius);
        j.kv("cutoff", T.ze_cutoff);
        j.close('}');
    }
    j.close(']');
    j.key("inverse_power");
    j.open('[');
    for (int k = 0; k < y.n_inverse_power; ++k) {
        const alea_gpu_inverse_power& V = y.inverse_power[k];
        j.open('{');
        j.arr("ga", std::vector<int>{V.a_first, V.a_last});
        j.arr("gb", std::vector<int>{V.b_first, V.b_last});
        j.kv("strength", V.strength);
        j.kv("exponent", V.exponent);
        j.kv("tail", V.tail);
        j.close('}');
    }
    j.close(']');
    if (!S->anchors.empty()) {
        j.arr("anchors", S->anchors);
        j.kv("jitter", S->jitter);
    }
    j.close('}');
    S->json = j.s;
}

void add_group(alea_gpu_system& y, int first, int n, double charge) {
    alea_gpu_group& g = y.groups[y.n_groups++];
    g.first = first;
    g.last = first + n;
    g.charge = charge;
    g.inv_mass[0] = g.inv_mass[1] = 1.0;
    g.inv_mass[2] = 0.0;
}

// Ewald tables into the system; returns (self, background) energies.
void add_ewald(alea_gpu_setup* S, const Cell& c, double tol, double& self, double& bg) {
    alea_gpu_system& y = S->sys;
    const Breakup br = ewald_breakup(c, tol);
    y.ewald.enabled = 1;
    y.ewald.r_cut = c.ws;
    y.ewald.inv_eps = 1.0;
    set_spline(S, y.ewald.long_range, br);
    set_kset(S, y.ewald.kset, br);
    double q2 = 0.0, Q = 0.0;
    for (int g = 0; g < y.n_groups; ++g) {
        const int n = y.groups[g].last - y.groups[g].first;
        q2 += y.groups[g].charge * y.groups[g].charge * n;
        Q += y.groups[g].charge * n;
    }
    self = -0.5 * br.long_range_zero * q2;
    bg = -0.5 * Q * Q * br.short_range_k0;
    y.ewald.constant = self + bg;
}

}  // namespace

extern "C" {

const alea_gpu_system* alea_gpu_setup_system(const alea_gpu_setup* s) { return s ? &s->sys : nullptr; }
const char* alea_gpu_setup_json(const alea_gpu_setup* s) { return s ? s->json.c_str() : ""; }
void alea_gpu_setup_free(alea_gpu_setup* s) { delete s; }

// 2-D homogeneous electron gas in a square cell of area N π r_s², plane-wave
// determinants per spin, image-summed Padé u = a₁ r/(1 + b r) on every spin
// pair (a₁ from the Kato cusp, or `pade_a` when positive for the opposite
// spins and half of it for equal spins), Ewald Coulomb.
static int setup_heg2d(int n_up, int n_down, double rs, double pade_b, double pade_a, double tx, double ty,
                       double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        if (n_up < 1 || n_down < 0 || !(rs > 0.0)) throw std::invalid_argument("heg2d: bad sizes");
        alea_gpu_system& y = S->sys;
        const int np = n_up + n_down;
        y.dim = 2;
        y.n_particles = np;
        y.periodic = 1;
        const double L = std::sqrt(np * kPi * rs * rs);
        const Cell c = make_cell(L, L);
        std::copy(c.a, c.a + 4, y.lattice);
        add_group(y, 0, n_up, -1.0);
        if (n_down > 0) add_group(y, n_up, n_down, -1.0);
        // an integer twist is Γ: the real closed-shell determinant
        const bool twisted = std::abs(tx - std::nearbyint(tx)) >= 1e-12 || std::abs(ty - std::nearbyint(ty)) >= 1e-12;
        for (int g = 0; g < y.n_groups; ++g) {
            std::vector<double> k;
            std::vector<int> is_sin;
            const int n = y.groups[g].last - y.groups[g].first;
            alea_gpu_orbitals& B = y.blocks[y.n_blocks++];
            B.first = y.groups[g].first;
            B.last = y.groups[g].last;
            if (twisted) {
                twisted_shells(c, n, tx, ty, k);
                B.type = ALEA_ORB_TWISTED_PLANE_WAVE;
                B.k = S->keep(k);
            } else {
                plane_wave_shells(c, n, k, is_sin);
                B.type = ALEA_ORB_PLANE_WAVE;
                B.k = S->keep(k);
                B.is_sin = S->keepi(is_sin);
            }
        }
        double self = 0.0, bg = 0.0;
        add_ewald(S, c, ewald_tol > 0.0 ? ewald_tol : 1e-6, self, bg);
        for (int ga = 0; ga < y.n_groups; ++ga)
            for (int gb = ga; gb < y.n_groups; ++gb) {
                const alea_gpu_group& A = y.groups[ga];
                const alea_gpu_group& B = y.groups[gb];
                if (ga == gb && A.last - A.first < 2) continue;
                const int ell = ga == gb ? 1 : 0;
                const double R = A.charge * B.charge;   // q_a q_b / ε
                double a1 = 2.0 * 0.5 * R / (2 * ell + 2 - 1);
                if (pade_a > 0.0) a1 = ga == gb ? 0.5 * pade_a : pade_a;
                alea_gpu_pair_term& T = y.terms[y.n_terms++];
                T.kind = ALEA_PAIR_PADE;
                T.n_pairs = 1;
                T.pairs[0][0] = A.first;
                T.pairs[0][1] = A.last;
                T.pairs[0][2] = B.first;
                T.pairs[0][3] = B.last;
                T.num_order = 1;
                T.den_order = 1;
                T.coeffs[0] = a1;
                T.coeffs[1] = pade_b;
                T.image_sum = 1;
                // equal-spin pairs share one table
                int same = -1;
                for (int q = 0; q + 1 < y.n_terms; ++q)
                    if (y.terms[q].coeffs[0] == a1) same = q;
                // the denominator b is the term's optimisable parameter (a_1 is
                // fixed by the cusp): the breakup of du/db = -a_1 r^2 / Q^2 on the
                // same options (src/wavefunction/pade_jastrow.cpp:214-248)
                T.n_opt = 1;
                T.opt_index[0] = 1;
                if (same >= 0) {
                    T.short_range = y.terms[same].short_range;
                    T.u_inf = y.terms[same].u_inf;
                    T.kset = y.terms[same].kset;
                    T.opt_inf[0] = y.terms[same].opt_inf[0];
                    T.opt_short_range[0] = y.terms[same].opt_short_range[0];
                    T.opt_weight[0] = y.terms[same].opt_weight[0];
                    continue;
                }
                double u_inf = 0.0;
                const Breakup br = pade_breakup(c, {a1}, {pade_b}, u_inf);
                set_spline(S, T.short_range, br);
                T.u_inf = u_inf;
                set_kset(S, T.kset, br);
                double d_inf = 0.0;
                const Breakup bp = pade_breakup(c, {0.0, -a1}, {2.0 * pade_b, pade_b * pade_b}, d_inf);
                if (bp.weight.size() != br.weight.size())
                    throw std::logic_error("heg2d: the parameter breakup's k set differs");
                T.opt_inf[0] = d_inf;
                set_spline(S, T.opt_short_range[0], bp);
                T.opt_weight[0] = S->keep(bp.weight);
            }
        write_json(S, "heg", self, bg);
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

int alea_gpu_setup_heg2d(int n_up, int n_down, double rs, double pade_b, double pade_a,
                         double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len) {
    return setup_heg2d(n_up, n_down, rs, pade_b, pade_a, 0.0, 0.0, ewald_tol, out, err, err_len);
}

int alea_gpu_setup_heg2d_twisted(int n_up, int n_down, double rs, double pade_b, double pade_a,
                                 double twist_x, double twist_y, double ewald_tol, alea_gpu_setup** out,
                                 char* err, size_t err_len) {
    return setup_heg2d(n_up, n_down, rs, pade_b, pade_a, twist_x, twist_y, ewald_tol, out, err, err_len);
}

// 2-D Wigner crystal: a triangular lattice of nx × ny sites (ny even) in the
// rectangular cell nx a × ny a √3/2 at density r_s, spin up on even rows and
// down on odd rows, Gaussian orbitals exp(−c |r − R|²) with c = gauss_c / r_s²,
// Drummond-Towler-Needs Jastrows (C = 3) with cutoff `cutoff_frac` × the
// Wigner-Seitz inradius and cusp-derived α₁ (same spins, opposite spins),
// Ewald Coulomb.  Initial walkers: sites + N(0, jitter).
int alea_gpu_setup_crystal2d(int nx, int ny, double rs, double gauss_c, double alpha0,
                             double cutoff_frac, double jitter, double ewald_tol,
                             alea_gpu_setup** out, char* err, size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        if (nx < 1 || ny < 2 || ny % 2 || !(rs > 0.0)) throw std::invalid_argument("crystal2d: bad sizes");
        alea_gpu_system& y = S->sys;
        const int N = nx * ny, nu = N / 2, nd = N - nu;
        y.dim = 2;
        y.n_particles = N;
        y.periodic = 1;
        const double alat = rs * std::sqrt(2.0 * kPi / std::sqrt(3.0));
        const double Lx = nx * alat, Ly = ny * alat * std::sqrt(3.0) / 2.0;
        const Cell c = make_cell(Lx, Ly);
        std::copy(c.a, c.a + 4, y.lattice);
        add_group(y, 0, nu, -1.0);
        add_group(y, nu, nd, -1.0);
        std::vector<double> up, dn;
        for (int r = 0; r < ny; ++r)
            for (int col = 0; col < nx; ++col) {
                auto& dst = (r % 2 == 0) ? up : dn;
                dst.push_back((col + 0.5 * (r % 2)) * alat - 0.5 * Lx);
                dst.push_back(r * alat * std::sqrt(3.0) / 2.0 - 0.5 * Ly);
            }
        const double alpha = gauss_c / (rs * rs);
        for (int g = 0; g < 2; ++g) {
            alea_gpu_orbitals& B = y.blocks[y.n_blocks++];
            B.first = y.groups[g].first;
            B.last = y.groups[g].last;
            B.type = ALEA_ORB_GAUSSIAN;
            B.centers = S->keep(g == 0 ? up : dn);
            B.alphas = S->keep(std::vector<double>(B.last - B.first, alpha));
        }
        S->anchors = up;
        S->anchors.insert(S->anchors.end(), dn.begin(), dn.end());
        S->jitter = jitter > 0.0 ? jitter : 1.0 / std::sqrt(4.0 * alpha);
        double self = 0.0, bg = 0.0;
        add_ewald(S, c, ewald_tol > 0.0 ? ewald_tol : 1e-6, self, bg);
        const double Lcut = (cutoff_frac > 0.0 ? cutoff_frac : 0.999) * c.ws;
        for (int item = 0; item < 2; ++item) {
            alea_gpu_pair_term& T = y.terms[y.n_terms++];
            T.kind = ALEA_PAIR_DRUMMOND;
            if (item == 0) {
                T.n_pairs = 2;
                for (int g = 0; g < 2; ++g) {
                    T.pairs[g][0] = T.pairs[g][2] = y.groups[g].first;
                    T.pairs[g][1] = T.pairs[g][3] = y.groups[g].last;
                }
            } else {
                T.n_pairs = 1;
                T.pairs[0][0] = y.groups[0].first;
                T.pairs[0][1] = y.groups[0].last;
                T.pairs[0][2] = y.groups[1].first;
                T.pairs[0][3] = y.groups[1].last;
            }
            T.C = 3;
            T.gamma = 2.0 * 0.5 * 1.0 / (2 * (item == 0 ? 1 : 0) + 1);
            T.L = Lcut;
            T.n_coeffs = 1;
            T.dcoeffs[0] = alpha0;
        }
        write_json(S, "crystal", self, bg);
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

// Point charges in a periodic 2-D cell with Ewald Coulomb only (no
// wavefunction factors, so E_L is the electrostatic energy): n_groups
// consecutive groups of counts[g] particles of charge charges[g].  The cell's
// rows are reduced as the device reduces them.  Initial walkers: uniform.
int alea_gpu_setup_charges2d(const double* lattice, int n_groups, const int* counts, const double* charges,
                             double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        if (!lattice || !counts || !charges || n_groups < 1 || n_groups > ALEA_GPU_MAX_GROUPS)
            throw std::invalid_argument("charges2d: bad groups");
        alea_gpu_system& y = S->sys;
        y.dim = 2;
        y.periodic = 1;
        const Cell c = make_cell(lattice);
        std::copy(c.a, c.a + 4, y.lattice);
        int first = 0;
        for (int g = 0; g < n_groups; ++g) {
            if (counts[g] < 1) throw std::invalid_argument("charges2d: empty group");
            add_group(y, first, counts[g], charges[g]);
            first += counts[g];
        }
        y.n_particles = first;
        double self = 0.0, bg = 0.0;
        add_ewald(S, c, ewald_tol > 0.0 ? ewald_tol : 1e-6, self, bg);
        write_json(S, "charges", self, bg);
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

// The 3-D Coulomb Ewald tables of a periodic cell (rows a_i of `lattice`, 9
// numbers): the optimized breakup of 1/r with the 3-D radial kernel
// 4π r sin(kr)/k, the knot count the smaller of 20, 24 whose shell misfit is
// below `ewald_tol`, r_c the Wigner-Seitz inradius (half the
// shortest lattice vector).  Host tables only (JSON: cell, the spline, the
// half-space k-vectors n1 n2 n3, kx ky kz with their weights, f_l(0) and
// f̃_s(0)/V); the walker kernels are two-dimensional.  No counterpart in the
// reference, which refuses 3-D Ewald (src/numerics/ewald_breakup.cpp:211-213).
}  // extern "C"

namespace {

// The optimized breakup of 1/r in a 3-D cell (rows a_i of `lattice`): the
// 3-D radial kernel, r_c the Wigner-Seitz inradius, the knot ladder 20, 24.
// In 3-D the misfit on the discrete shells understates the energy's error
// (the neglected tail grows with the k² density of vectors): 12 knots pass a
// 1e-10 shell tolerance yet leave 2e-7 in the CsCl Madelung constant, 20
// knots 7e-9.  The ladder starts at 20.
Breakup ewald3d_breakup(const double* lattice, double ewald_tol, double& rc, double& volume) {
    if (!lattice) throw std::invalid_argument("ewald3d: no lattice");
    alea_breakup::Lattice lat;
    lat.dim = 3;
    std::copy(lattice, lattice + 9, lat.a);
    const double* a = lat.a;
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (det == 0.0 || !std::isfinite(det)) throw std::invalid_argument("ewald3d: singular lattice vectors");
    lat.volume = std::abs(det);
    // b_i · a_j = 2π δ_ij: b = 2π (Aᵀ)⁻¹, rows b_i
    const double inv[9] = {(a[4] * a[8] - a[5] * a[7]) / det, (a[2] * a[7] - a[1] * a[8]) / det,
                           (a[1] * a[5] - a[2] * a[4]) / det, (a[5] * a[6] - a[3] * a[8]) / det,
                           (a[0] * a[8] - a[2] * a[6]) / det, (a[2] * a[3] - a[0] * a[5]) / det,
                           (a[3] * a[7] - a[4] * a[6]) / det, (a[1] * a[6] - a[0] * a[7]) / det,
                           (a[0] * a[4] - a[1] * a[3]) / det};
    for (int i = 0; i < 3; ++i)
        for (int d = 0; d < 3; ++d) lat.b[i * 3 + d] = kTwoPi * inv[d * 3 + i];
    double shortest2 = 0.0;
    for (int n0 = -2; n0 <= 2; ++n0)
        for (int n1 = -2; n1 <= 2; ++n1)
            for (int n2 = -2; n2 <= 2; ++n2) {
                if (!n0 && !n1 && !n2) continue;
                double r2 = 0.0;
                for (int d = 0; d < 3; ++d) {
                    const double x = n0 * a[d] + n1 * a[3 + d] + n2 * a[6 + d];
                    r2 += x * x;
                }
                if (shortest2 == 0.0 || r2 < shortest2) shortest2 = r2;
            }
    rc = 0.5 * std::sqrt(shortest2);
    volume = lat.volume;
    const double tol = ewald_tol > 0.0 ? ewald_tol : 1e-6;
    const auto f = alea_breakup::coulomb();
    for (int nk : {20, 24}) {
        alea_breakup::Options opt;
        opt.n_knots = nk;
        Breakup br = alea_breakup::optimize(lat, rc, *f, opt);
        if (br.residual < tol) return br;
    }
    throw std::runtime_error("ewald3d: the breakup did not reach the requested tolerance");
}

void json_ewald3d(Json& j, double rc, const Breakup& br) {
    j.key("ewald");
    j.open('{');
    j.kv("r_cut", rc);
    j.key("spline");
    j.open('{');
    j.kv("r_cut", br.rc);
    j.kv("inv_delta", 1.0 / br.delta);
    j.kv("n_knots", br.n_knots);
    j.arr("scaled", br.scaled);
    j.close('}');
    j.arr("n1", br.n[0]);
    j.arr("n2", br.n[1]);
    j.arr("n3", br.n[2]);
    j.arr("kx", br.kvec[0]);
    j.arr("ky", br.kvec[1]);
    j.arr("kz", br.kvec[2]);
    j.arr("weight", br.weight);
    j.kv("v_long_zero", br.long_range_zero);
    j.kv("sr_k0", br.short_range_k0);
    j.kv("residual", br.residual);
}

// Real 3-D plane waves of the lowest shells of a cubic cell of side L: k =
// 2π n / L with n sorted by |n|², then lexicographically; k = 0 gives
// cos(0), every other ±n pair is represented by the n whose first nonzero
// component is positive and gives cos then sin.
void plane_waves_3d(double L, int n, std::vector<double>& k, std::vector<int>& is_sin) {
    std::vector<std::array<int, 4>> cand;
    for (int a = -4; a <= 4; ++a)
        for (int b = -4; b <= 4; ++b)
            for (int c = -4; c <= 4; ++c) {
                const int first = a != 0 ? a : (b != 0 ? b : c);
                if (first < 0) continue;
                cand.push_back({a * a + b * b + c * c, a, b, c});
            }
    std::sort(cand.begin(), cand.end());
    k.clear();
    is_sin.clear();
    for (const auto& q : cand) {
        if (static_cast<int>(is_sin.size()) >= n) break;
        for (int s = 0; s < (q[0] == 0 ? 1 : 2) && static_cast<int>(is_sin.size()) < n; ++s) {
            for (int d = 0; d < 3; ++d) k.push_back(kTwoPi * q[1 + d] / L);
            is_sin.push_back(s);
        }
    }
    if (static_cast<int>(is_sin.size()) != n) throw std::invalid_argument("heg3d: too many electrons per spin");
}

}  // namespace

extern "C" {

int alea_gpu_setup_ewald3d(const double* lattice, double ewald_tol, alea_gpu_setup** out, char* err,
                           size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        double rc = 0.0, volume = 0.0;
        const Breakup br = ewald3d_breakup(lattice, ewald_tol, rc, volume);
        S->sys.dim = 3;
        S->sys.periodic = 1;
        Json j;
        j.open('{');
        j.ks("kind", "ewald3d");
        j.kv("dim", 3);
        j.key("cell");
        j.open('{');
        j.arr("vectors", std::vector<double>(lattice, lattice + 9));
        j.kv("volume", volume);
        j.close('}');
        json_ewald3d(j, rc, br);
        j.close('}');
        j.close('}');
        S->json = j.s;
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

// 3-D electron gas with backflow: n_up + n_down electrons in a cubic cell of
// volume N 4π r_s³ / 3, one backflow determinant of real plane waves per spin
// (plane_waves_3d; every spin must close its shell), channels from the own
// spin (c_0 = bf_like, c_1 = 3 c_0 / L: zero slope) and the other spin
// (c_0 = bf_unlike, c_1 = 0), C = 3, L = bf_cut (<= 0: half the side);
// Drummond Jastrows (C = 3, the 3-D Kato cusps 1/2 and 1/4, alpha0, cutoff
// 0.999 × half the side) on the like-spin pairs and the unlike pair; the 3-D
// Ewald sum.  Initial walkers: uniform.
int alea_gpu_setup_heg3d(int n_up, int n_down, double rs, double bf_like, double bf_unlike, double bf_cut,
                         double alpha0, double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        if (n_up < 1 || n_down < 1 || n_up > 64 || n_down > 64 || !(rs > 0.0))
            throw std::invalid_argument("heg3d: need 1..64 electrons per spin and rs > 0");
        alea_gpu_system& y = S->sys;
        const int np = n_up + n_down;
        const double L = rs * std::cbrt(4.0 * kPi * np / 3.0);
        y.dim = 3;
        y.n_particles = np;
        y.periodic = 1;
        const double lat[9] = {L, 0, 0, 0, L, 0, 0, 0, L};
        std::copy(lat, lat + 9, y.lattice);
        for (int g = 0; g < 2; ++g) {
            alea_gpu_group& G = y.groups[y.n_groups++];
            G.first = g == 0 ? 0 : n_up;
            G.last = g == 0 ? n_up : np;
            G.charge = -1.0;
            G.inv_mass[0] = G.inv_mass[1] = G.inv_mass[2] = 1.0;
        }
        const double Lb = bf_cut > 0.0 ? bf_cut : 0.5 * L;
        if (Lb > 0.5 * L) throw std::invalid_argument("heg3d: the backflow cutoff exceeds half the cell");
        y.n_backflow = 2;
        for (int g = 0; g < 2; ++g) {
            alea_gpu_backflow& F = y.backflow[g];
            F.first = y.groups[g].first;
            F.last = y.groups[g].last;
            F.type = ALEA_ORB_PLANE_WAVE;
            std::vector<double> k;
            std::vector<int> is_sin;
            plane_waves_3d(L, F.last - F.first, k, is_sin);
            F.k = S->keep(k);
            F.is_sin = S->keepi(is_sin);
            F.n_channels = 2;
            for (int h = 0; h < 2; ++h) {
                alea_gpu_backflow_channel& C = F.channels[h];
                C.source_first = y.groups[h].first;
                C.source_last = y.groups[h].last;
                C.C = 3;
                C.L = Lb;
                C.n_coeffs = 2;
                C.coeffs[0] = h == g ? bf_like : bf_unlike;
                C.coeffs[1] = h == g ? 3.0 * bf_like / Lb : 0.0;
                C.zero_slope = h == g ? 1 : 0;
            }
        }
        const double Lj = 0.999 * 0.5 * L;
        y.n_terms = 2;
        for (int t = 0; t < 2; ++t) {
            alea_gpu_pair_term& T = y.terms[t];
            T.kind = ALEA_PAIR_DRUMMOND;
            if (t == 0) {
                T.n_pairs = 2;
                const int pr[2][4] = {{0, n_up, 0, n_up}, {n_up, np, n_up, np}};
                for (int q = 0; q < 2; ++q)
                    for (int c = 0; c < 4; ++c) T.pairs[q][c] = pr[q][c];
                T.gamma = 0.25;
            } else {
                T.n_pairs = 1;
                const int pr[4] = {0, n_up, n_up, np};
                for (int c = 0; c < 4; ++c) T.pairs[0][c] = pr[c];
                T.gamma = 0.5;
            }
            T.C = 3;
            T.L = Lj;
            T.n_coeffs = 1;
            T.dcoeffs[0] = alpha0;
        }
        double rc = 0.0, volume = 0.0;
        const Breakup br = ewald3d_breakup(lat, ewald_tol, rc, volume);
        alea_gpu_ewald& E = y.ewald;
        E.enabled = 1;
        E.r_cut = rc;
        E.inv_eps = 1.0;
        set_spline(S, E.long_range, br);
        E.kset.n_k = static_cast<int>(br.weight.size());
        E.kset.n1 = S->keepi(br.n[0]);
        E.kset.n2 = S->keepi(br.n[1]);
        E.kset.n3 = S->keepi(br.n[2]);
        E.kset.kx = S->keep(br.kvec[0]);
        E.kset.ky = S->keep(br.kvec[1]);
        E.kset.kz = S->keep(br.kvec[2]);
        E.kset.weight = S->keep(br.weight);
        const double self = -0.5 * br.long_range_zero * np, bg = -0.5 * double(np) * np * br.short_range_k0;
        E.constant = self + bg;
        Json j;
        j.open('{');
        j.ks("kind", "heg3d");
        j.kv("dim", 3);
        j.kv("np", np);
        j.key("cell");
        j.open('{');
        j.kv("periodic", 1);
        j.kv("dim", 3);
        j.arr("vectors", std::vector<double>(lat, lat + 9));
        j.close('}');
        j.key("groups");
        j.open('[');
        for (int g = 0; g < 2; ++g) {
            j.open('{');
            j.kv("first", y.groups[g].first);
            j.kv("last", y.groups[g].last);
            j.kv("charge", -1.0);
            j.arr("inv_mass", std::vector<double>{1.0, 1.0, 1.0});
            j.close('}');
        }
        j.close(']');
        j.key("backflow");
        j.open('[');
        for (int g = 0; g < 2; ++g) {
            const alea_gpu_backflow& F = y.backflow[g];
            const int n = F.last - F.first;
            j.open('{');
            j.kv("first", F.first);
            j.kv("last", F.last);
            j.ks("type", "plane_wave");
            j.arr("k", std::vector<double>(F.k, F.k + 3 * n));
            j.arr("is_sin", std::vector<int>(F.is_sin, F.is_sin + n));
            j.key("channels");
            j.open('[');
            for (int h = 0; h < 2; ++h) {
                const alea_gpu_backflow_channel& C = F.channels[h];
                j.open('{');
                j.kv("source_first", C.source_first);
                j.kv("source_last", C.source_last);
                j.kv("C", C.C);
                j.arr("coeffs", std::vector<double>(C.coeffs, C.coeffs + C.n_coeffs));
                j.kv("L", C.L);
                j.kv("zero_slope", C.zero_slope);
                j.close('}');
            }
            j.close(']');
            j.close('}');
        }
        j.close(']');
        j.key("drummond");
        j.open('[');
        for (int t = 0; t < 2; ++t) {
            const alea_gpu_pair_term& T = y.terms[t];
            j.open('{');
            j.kv("C", T.C);
            j.kv("gamma", T.gamma);
            j.kv("L", T.L);
            j.arr("coeffs", std::vector<double>{alpha0});
            j.key("pairs");
            j.open('[');
            for (int q = 0; q < T.n_pairs; ++q) j.arr("", std::vector<int>(T.pairs[q], T.pairs[q] + 4));
            j.close(']');
            j.close('}');
        }
        j.close(']');
        json_ewald3d(j, rc, br);
        j.kv("inv_eps", 1.0);
        j.kv("self_energy", self);
        j.kv("background_energy", bg);
        j.close('}');
        j.close('}');
        S->json = j.s;
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

// 2-D dipolar bosons (the reference's configs/dipoles_2d_gas_n256.yaml
// shape): n bosons of mass 1 in a hexagonal cell of area n π rs²
// (app.cpp:314-330), C r^-p at the minimum image plus the continuum tail
// outside the Wigner-Seitz cell (inverse_power.cpp:28-80), and the
// zero-energy Jastrow with b = 2 μ C, μ = 1/2, cut off at the Wigner-Seitz
// inradius (builders/jastrow.cpp:202-260).  Initial walkers: uniform.
int alea_gpu_setup_dipoles2d(int n, double rs, double strength, double exponent, double matching_radius,
                             alea_gpu_setup** out, char* err, size_t err_len) {
    if (!out) return ALEA_ERR_INVALID;
    *out = nullptr;
    auto* S = new alea_gpu_setup();
    try {
        if (n < 2 || !(rs > 0.0) || !(exponent > 2.0) || !(strength > 0.0))
            throw std::invalid_argument("dipoles2d: needs n >= 2, rs > 0, strength > 0, exponent > 2");
        alea_gpu_system& y = S->sys;
        y.dim = 2;
        y.n_particles = n;
        y.periodic = 1;
        const double area = n * kPi * rs * rs;
        const double L = std::sqrt(2.0 * area / std::sqrt(3.0));
        const double lat[4] = {L, 0.0, 0.5 * L, L * std::sqrt(3.0) / 2.0};
        const Cell c = make_cell(lat);
        std::copy(c.a, c.a + 4, y.lattice);
        add_group(y, 0, n, 0.0);
        if (!(matching_radius > 0.0 && matching_radius < c.ws))
            throw std::invalid_argument("dipoles2d: the matching radius must lie inside (0, r_WS = " +
                                        std::to_string(c.ws) + ")");
        alea_gpu_pair_term& T = y.terms[y.n_terms++];
        T.kind = ALEA_PAIR_ZERO_ENERGY;
        T.n_pairs = 1;
        T.pairs[0][0] = T.pairs[0][2] = 0;
        T.pairs[0][1] = T.pairs[0][3] = n;
        T.ze_b = 2.0 * 0.5 * strength;
        T.ze_exponent = exponent;
        T.ze_matching_radius = matching_radius;
        T.ze_cutoff = c.ws;
        alea_gpu_inverse_power& V = y.inverse_power[y.n_inverse_power++];
        V.a_first = V.b_first = 0;
        V.a_last = V.b_last = n;
        V.strength = strength;
        V.exponent = exponent;
        const double outside =
            ws_exterior_integral(c, [&](double rho) { return std::pow(rho, 2.0 - exponent); }) /
            (exponent - 2.0);
        const double pairs = 0.5 * static_cast<double>(n) * static_cast<double>(n);
        V.tail = pairs / c.area * strength * outside;
        write_json(S, "dipoles", 0.0, 0.0);
    } catch (const std::exception& e) {
        if (err && err_len) std::snprintf(err, err_len, "%s", e.what());
        delete S;
        return ALEA_ERR_INVALID;
    }
    *out = S;
    return ALEA_OK;
}

// Open 2-D exciton: electron and hole, exact trial u = −r (Padé with the
// Kato cusp a₁ = −1), open Coulomb −1/r.  E = −1 with zero variance.
int alea_gpu_setup_exciton2d(double L_init, alea_gpu_setup** out) {
    if (!out) return ALEA_ERR_INVALID;
    auto* S = new alea_gpu_setup();
    alea_gpu_system& y = S->sys;
    y.dim = 2;
    y.n_particles = 2;
    y.periodic = 0;
    add_group(y, 0, 1, -1.0);
    add_group(y, 1, 1, 1.0);
    alea_gpu_pair_term& T = y.terms[y.n_terms++];
    T.kind = ALEA_PAIR_PADE;
    T.n_pairs = 1;
    T.pairs[0][0] = 0;
    T.pairs[0][1] = 1;
    T.pairs[0][2] = 1;
    T.pairs[0][3] = 2;
    T.num_order = 1;
    T.den_order = 0;
    T.coeffs[0] = 2.0 * 0.5 * (-1.0) / 1.0;
    alea_gpu_coulomb& C = y.coulomb[y.n_coulomb++];
    C.a_first = 0;
    C.a_last = 1;
    C.b_first = 1;
    C.b_last = 2;
    C.coef = -1.0;
    S->open_L = L_init > 0.0 ? L_init : 1.0;
    write_json(S, "exciton", 0.0, 0.0);
    *out = S;
    return ALEA_OK;
}

// Initial positions with the reference App's semantics (app.cpp:56-112):
// one mt19937_64 seeded with `seed`, walkers in order, particles in order;
// uniform fractional coordinates in [−½, ½) through the cell vectors, uniform
// in [−L/2, L/2) for an open cell, or site + jitter × N(0, 1) for a crystal.
// lo + (hi − lo) u and the lattice sums are fused multiply-adds, the rounding
// of the reference built with FMA contraction.  positions: AoS [w][p][d].
int alea_gpu_setup_positions(const alea_gpu_setup* S, uint64_t seed, int nw, double* positions) {
    if (!S || !positions || nw < 0) return ALEA_ERR_INVALID;
    const alea_gpu_system& y = S->sys;
    std::mt19937_64 eng(seed);
    std::uniform_real_distribution<double> uni(0.0, 1.0);
    std::normal_distribution<double> gau(0.0, 1.0);
    const int np = y.n_particles, dim = y.dim;
    for (int w = 0; w < nw; ++w)
        for (int p = 0; p < np; ++p) {
            double* r = positions + (static_cast<size_t>(w) * np + p) * dim;
            if (!S->anchors.empty()) {
                for (int d = 0; d < dim; ++d) r[d] = std::fma(S->jitter, gau(eng), S->anchors[p * dim + d]);
            } else if (y.periodic) {
                double f[3];
                for (int i = 0; i < dim; ++i) f[i] = std::fma(1.0, uni(eng), -0.5);
                for (int d = 0; d < dim; ++d) {
                    double acc = 0.0;
                    for (int i = 0; i < dim; ++i) acc = std::fma(f[i], y.lattice[i * dim + d], acc);
                    r[d] = acc;
                }
            } else {
                for (int d = 0; d < dim; ++d) r[d] = std::fma(S->open_L, uni(eng), -0.5 * S->open_L);
            }
        }
    return ALEA_OK;
}

}  // extern "C"
