// Test-infrastructure driver for the reference implementation.
//
// Compiled by oracle/Makefile together with the reference's own hot-path
// sources (read in place from the reference tree) into oracle/_ref/ref_harness.
// It never enters the product: the tests use it to pin the oracle restatement
// and to produce golden fixtures, and bench.py's reference arm uses it as the
// CPU baseline.  It builds the same objects the reference's App builds for a
// YAML config (src/qmc/app.cpp:432-452 Hamiltonian order, src/builders/
// jastrow.cpp:48-63 cusps, :339-389 image-summed Padé under Ewald,
// src/builders/slater.cpp:267 plane-wave shells), but directly, without the
// YAML/HDF5 layers, the way tests/test_dmc_bench.cpp does.
//
// usage: ref_harness MODE key=value...
//   MODE setup  : print the system description (every setup-time table) as JSON
//   MODE init   : print the initial walker positions (app.cpp:56-112 semantics)
//   MODE eval   : evaluate ln|psi|, grad, lap and E_L of the initial walkers
//   MODE vmc    : run the reference VMC driver and print its trace
//   MODE dmc    : run the reference DMC driver and print its trace
//   MODE bench  : time DMC (or VMC, method=vmc) steps with all host threads
//   MODE chain  : VMC, then DMC seeded from VMC's final configurations
//   MODE estimate : accumulate the estimators (gofr / density / sofk) over
//                   fixed configurations with given weights, print their series
//   MODE gpu_pair : (ref_harness_gpu only, built with the reference-side GPU
//                   drivers of alea_b200/adapter) the reference's VMC or DMC
//                   (method=vmc|dmc) and GpuVMC / GpuDMC on copies of the same
//                   ensemble, the system flattened by alea::gpu::pack_system
//                   from the objects built here; both traces printed
// Every mode takes pos_file=PATH (whitespace-separated AoS positions of the nw
// walkers) in place of the seeded initialisation.
// vmc and dmc attach the same estimators when gofr_bins, dens_bins or
// sofk_kmax is given, and print the estimators' series of run_result().
#include <omp.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "estimators/density.h"
#include "estimators/pair_correlation.h"
#include "estimators/structure_factor.h"
#include "hamiltonian/coulomb.h"
#include "hamiltonian/ewald_term.h"
#include "hamiltonian/inverse_power.h"
#include "hamiltonian/hamiltonian.h"
#include "hamiltonian/kinetic.h"
#include "numerics/long_range_breakup.h"
#include "numerics/pair_radial.h"
#include "numerics/random.h"
#include "numerics/xoshiro_random.h"
#include "population/walker.h"
#include "population/walker_ensemble.h"
#include "population/walker_set.h"
#include "qmc/dmc.h"
#include "qmc/vmc.h"
#include "wavefunction/backflow_slater_determinant.h"
#include "wavefunction/complex_orbital_set.h"
#include "wavefunction/complex_slater_determinant.h"
#include "wavefunction/drummond_jastrow.h"
#include "wavefunction/orbital_set.h"
#include "wavefunction/pade_jastrow.h"
#include "wavefunction/slater_determinant.h"
#include "wavefunction/trial_wavefunction.h"
#include "wavefunction/zero_energy_jastrow.h"

#ifdef ALEA_GPU_DRIVER
#include "../alea_b200/adapter/alea_gpu_driver.h"
#endif

using namespace alea;

namespace {

// ── tiny JSON writer ────────────────────────────────────────────────────────
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
        if (std::isfinite(x))
            std::snprintf(b, sizeof b, "%.17g", x);
        else
            std::snprintf(b, sizeof b, "null");
        s += b;
    }
    void inum(long long x) {
        sep();
        s += std::to_string(x);
    }
    void str(const std::string& x) {
        sep();
        s += "\"" + x + "\"";
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
        key(k);
        open('[');
        for (auto x : v) num(static_cast<double>(x));
        close(']');
    }
    void kv(const std::string& k, double x) {
        key(k);
        num(x);
    }
    void ki(const std::string& k, long long x) {
        key(k);
        inum(x);
    }
    void ks(const std::string& k, const std::string& x) {
        key(k);
        str(x);
    }
};

using Args = std::map<std::string, std::string>;

double getd(const Args& a, const std::string& k, double d) {
    auto it = a.find(k);
    return it == a.end() ? d : std::stod(it->second);
}
long long geti(const Args& a, const std::string& k, long long d) {
    auto it = a.find(k);
    return it == a.end() ? d : std::stoll(it->second);
}
std::string gets(const Args& a, const std::string& k, const std::string& d) {
    auto it = a.find(k);
    return it == a.end() ? d : it->second;
}

ParticleGroup make_group(const std::string& name, std::size_t first, std::size_t n,
                         double charge, std::size_t dim, double mass = 1.0) {
    ParticleGroup g;
    g.name = name;
    g.mass.assign(dim, mass);
    g.inv_mass.assign(dim, 1.0 / mass);
    g.charge = charge;
    g.first = first;
    g.last = first + n;
    g.count = n;
    return g;
}

// Everything one system needs, plus what the setup dump reports.
struct System {
    std::string kind;
    std::size_t dim = 2, np = 0;
    std::vector<ParticleGroup> groups;
    SimulationCell cell;
    TrialWavefunction psi;
    Hamiltonian ham;
    double L_open = 1.0;                 // open-cell initialisation box
    std::vector<double> anchors;         // [np*dim] crystal sites per particle
    double jitter = 0.0;
    Json setup;                          // system description
#ifdef ALEA_GPU_DRIVER
    std::vector<gpu::PadeTermSpec> pade_specs;   // what pack_system cannot read off a PadeJastrow
#endif
};

void dump_cell(Json& j, const SimulationCell& c) {
    j.key("cell");
    j.open('{');
    j.ki("periodic", c.is_periodic() ? 1 : 0);
    j.ki("dim", static_cast<long long>(c.dim()));
    if (c.is_periodic()) {
        j.arr("vectors", c.vectors());
        j.arr("reciprocal", c.reciprocal());
        j.ki("orthorhombic", c.orthorhombic() ? 1 : 0);
        j.kv("volume", c.volume());
        j.kv("ws_radius", c.ws_radius());
    }
    j.close('}');
}

void dump_groups(Json& j, const std::vector<ParticleGroup>& groups) {
    j.key("groups");
    j.open('[');
    for (const ParticleGroup& g : groups) {
        j.open('{');
        j.ks("name", g.name);
        j.ki("first", static_cast<long long>(g.first));
        j.ki("last", static_cast<long long>(g.last));
        j.kv("charge", g.charge);
        j.arr("inv_mass", g.inv_mass);
        j.close('}');
    }
    j.close(']');
}

void dump_spline(Json& j, const std::string& k, const numerics::LongRangeSpline& sp) {
    j.key(k);
    j.open('{');
    j.kv("r_cut", sp.r_cut);
    j.kv("inv_delta", sp.inv_delta);
    j.ki("n_knots", sp.n_knots);
    j.arr("scaled", sp.scaled);
    j.close('}');
}

// The image-summed Padé tables, rebuilt with exactly the calls and options of
// PeriodicPairSum's constructor (src/wavefunction/periodic_pair_sum.cpp:21-60),
// which is deterministic: same inputs, same tables.
void dump_pade_image_sum(Json& j, const SimulationCell& cell, const std::vector<double>& a,
                         const std::vector<double>& b) {
    const double rc = cell.ws_radius();
    numerics::BreakupOptions opt{};
    opt.k_continuum = 20.0 * 3.14159265358979323846 / rc;
    opt.k_max = 300.0 / rc;
    opt.n_continuum = 150;
    opt.k_cut = 5.0 * std::min(std::hypot(cell.reciprocal()[0], cell.reciprocal()[1]),
                               std::hypot(cell.reciprocal()[2], cell.reciprocal()[3]));
    const numerics::LongRangeBreakup br =
        numerics::build_long_range_breakup(cell, numerics::pade_radial(a, b, rc), opt);
    j.key("image_sum");
    j.open('{');
    dump_spline(j, "spline", br.spline());
    j.kv("u_inf", numerics::pade_limit(a, b));
    j.arr("n1", br.n1());
    j.arr("n2", br.n2());
    j.arr("kx", br.kx());
    j.arr("ky", br.ky());
    j.arr("weight", br.weight());
    j.kv("k_cut", br.k_cut());
    j.close('}');
}

// The optimisable parameters' breakups of an image-summed Padé, with the
// calls of PadeJastrow::build_image_sum (src/wavefunction/pade_jastrow.cpp:
// 214-248): du/da_k = r^k/Q, du/db_k = -P r^k/Q^2, each split on the same
// options.  free[i] marks parameter i of [a_1..a_N, b_1..b_M] as optimisable.
void dump_pade_opt(Json& j, const SimulationCell& cell, const std::vector<double>& a,
                   const std::vector<double>& b, const std::vector<bool>& free) {
    const double rc = cell.ws_radius();
    numerics::BreakupOptions opt{};
    opt.k_continuum = 20.0 * 3.14159265358979323846 / rc;
    opt.k_max = 300.0 / rc;
    opt.n_continuum = 150;
    opt.k_cut = 5.0 * std::min(std::hypot(cell.reciprocal()[0], cell.reciprocal()[1]),
                               std::hypot(cell.reciprocal()[2], cell.reciprocal()[3]));
    std::vector<double> q2(2 * b.size(), 0.0);
    for (std::size_t jj = 0; jj < b.size(); ++jj) {
        q2[jj] += 2.0 * b[jj];
        for (std::size_t l = 0; l < b.size(); ++l) q2[jj + l + 1] += b[jj] * b[l];
    }
    j.key("opt");
    j.open('[');
    for (std::size_t i = 0; i < free.size(); ++i) {
        if (!free[i]) continue;
        std::vector<double> num, den;
        if (i < a.size()) {
            num.assign(i + 1, 0.0);
            num[i] = 1.0;
            den = b;
        } else {
            const std::size_t k = i - a.size() + 1;
            num.assign(a.size() + k, 0.0);
            for (std::size_t jj = 0; jj < a.size(); ++jj) num[jj + k] = -a[jj];
            den = q2;
        }
        const numerics::LongRangeBreakup bp =
            numerics::build_long_range_breakup(cell, numerics::pade_radial(num, den, rc), opt);
        j.open('{');
        j.ki("index", static_cast<long long>(i));
        j.kv("inf", numerics::pade_limit(num, den));
        dump_spline(j, "spline", bp.spline());
        j.arr("weight", bp.weight());
        j.close('}');
    }
    j.close(']');
}

// ── systems ─────────────────────────────────────────────────────────────────

// 2D homogeneous electron gas: plane-wave determinants per spin, image-summed
// Padé u = a1 r/(1 + b r) on every spin pair (a1 from the Kato cusp), Ewald.
std::unique_ptr<System> build_heg(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "heg";
    const std::size_t nu = static_cast<std::size_t>(geti(a, "nu", 21));
    const std::size_t nd = static_cast<std::size_t>(geti(a, "nd", 21));
    const double rs = getd(a, "rs", 30.0);
    const double bden = getd(a, "b", 0.3);
    const double tol = getd(a, "tol", 1e-6);
    const double pi = 3.14159265358979323846;
    s->dim = 2;
    s->np = nu + nd;
    const double L = std::sqrt(static_cast<double>(s->np) * pi * rs * rs);
    const std::vector<double> vec{L, 0.0, 0.0, L};
    s->cell = SimulationCell(2, vec);
    s->groups.push_back(make_group("up", 0, nu, -1.0, 2));
    if (nd > 0) s->groups.push_back(make_group("down", nu, nd, -1.0, 2));

    // Hamiltonian: kinetic, then one cell-wide Ewald term (app.cpp:438-445).
    s->ham.add_component(std::make_unique<Kinetic>(s->groups));
    auto ewald = std::make_unique<EwaldTerm>(s->groups, 1.0, s->cell, tol);
    const EwaldTerm& ew = *ewald;

    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "heg");
    j.ki("dim", 2);
    j.ki("np", static_cast<long long>(s->np));
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);

    // Twisted boundary conditions (builders/slater.cpp:244-262): twisted plane
    // waves e^{i(k+θ)·r}, θ = t1 b1 + t2 b2, in a complex determinant.
    const std::vector<double> twist{getd(a, "tx", 0.0), getd(a, "ty", 0.0)};
    const bool twisted = std::abs(twist[0] - std::nearbyint(twist[0])) >= 1e-12 ||
                         std::abs(twist[1] - std::nearbyint(twist[1])) >= 1e-12;
    if (twisted) {
        std::vector<ComplexSlaterDeterminant::Block> cblocks;
        j.key("slater");
        j.open('[');
        for (const ParticleGroup& g : s->groups) {
            auto orb = make_twisted_plane_wave_orbitals(s->cell, g.size(), twist);
            j.open('{');
            j.ki("first", static_cast<long long>(g.first));
            j.ki("last", static_cast<long long>(g.last));
            j.ks("type", "twisted_plane_wave");
            const auto q = orb->wavevectors();
            j.arr("q", std::vector<double>(q.begin(), q.end()));
            j.arr("twist", twist);
            j.close('}');
            cblocks.push_back({g.first, g.last, std::move(orb)});
        }
        j.close(']');
        s->psi.add_component(std::make_unique<ComplexSlaterDeterminant>(std::move(cblocks)));
    }
    // Backflow (builders/slater.cpp:117-167): one backflow determinant per
    // spin group (one plane-wave block), channels from the own group (like
    // spin, c_1 derived) and from the other group, C = 3, L = the Wigner-Seitz
    // inradius.
    const bool backflow = geti(a, "bf", 0) != 0;
    if (backflow && !twisted) {
        const double c_like = getd(a, "bf_like", 0.3);
        const double c_un0 = getd(a, "bf_un0", 0.2), c_un1 = getd(a, "bf_un1", 0.002);
        const double L = s->cell.ws_radius();
        j.key("backflow");
        j.open('[');
        for (std::size_t gi = 0; gi < s->groups.size(); ++gi) {
            const ParticleGroup& g = s->groups[gi];
            auto orb = make_plane_wave_orbitals(s->cell, g.size());
            j.open('{');
            j.ki("first", static_cast<long long>(g.first));
            j.ki("last", static_cast<long long>(g.last));
            j.ks("type", "plane_wave");
            j.arr("k", orb->kvectors());
            const ReciprocalShellTable t = reciprocal_shell_table(s->cell, g.size());
            std::vector<double> is_sin(t.is_sin.begin(), t.is_sin.begin() + g.size());
            j.arr("is_sin", is_sin);
            std::vector<BackflowSlaterDeterminant::Channel> chans;
            j.key("channels");
            j.open('[');
            for (std::size_t hi = 0; hi < s->groups.size(); ++hi) {
                const ParticleGroup& h = s->groups[hi];
                BackflowSlaterDeterminant::Channel ch;
                ch.source_first = h.first;
                ch.source_last = h.last;
                ch.truncation = 3;
                std::vector<double> full;   // c_0 .. c_N as BackflowFunction holds them
                if (hi == gi) {
                    ch.params = {Parameter{"", c_like, false}, Parameter{"", L, true}};
                    full = {c_like, 3.0 * c_like / L};
                } else {
                    ch.params = {Parameter{"", c_un0, false}, Parameter{"", c_un1, false},
                                 Parameter{"", L, true}};
                    full = {c_un0, c_un1};
                }
                j.open('{');
                j.ki("source_first", static_cast<long long>(h.first));
                j.ki("source_last", static_cast<long long>(h.last));
                j.ki("C", 3);
                j.arr("coeffs", full);
                j.kv("L", L);
                // free parameters in BackflowFunction's order [c_0, (c_1), .., L]
                j.ki("zero_slope", hi == gi ? 1 : 0);
                std::vector<double> opt;
                for (std::size_t q = 0; q < ch.params.size(); ++q)
                    if (!ch.params[q].is_fixed) opt.push_back(static_cast<double>(q));
                j.arr("opt_index", opt);
                j.close('}');
                chans.push_back(std::move(ch));
            }
            j.close(']');
            j.close('}');
            std::vector<BackflowSlaterDeterminant::Block> bb;
            bb.push_back({g.first, g.last, std::move(orb)});
            s->psi.add_component(std::make_unique<BackflowSlaterDeterminant>(
                std::move(bb), std::move(chans), s->cell));
        }
        j.close(']');
    }
    // Slater: one plane-wave block per spin group (builders/slater.cpp:267).
    std::vector<SlaterDeterminant::Block> blocks;
    const bool plain = !twisted && !backflow;
    if (plain) j.key("slater");
    if (plain) j.open('[');
    for (const ParticleGroup& g : s->groups) {
        if (!plain) break;
        auto orb = make_plane_wave_orbitals(s->cell, g.size());
        j.open('{');
        j.ki("first", static_cast<long long>(g.first));
        j.ki("last", static_cast<long long>(g.last));
        j.ks("type", "plane_wave");
        j.arr("k", orb->kvectors());
        // is_sin is private; recover it from the shell table the factory used.
        const ReciprocalShellTable t = reciprocal_shell_table(s->cell, g.size());
        std::vector<double> is_sin(t.is_sin.begin(), t.is_sin.begin() + g.size());
        j.arr("is_sin", is_sin);
        j.close('}');
        blocks.push_back({g.first, g.last, std::move(orb)});
    }
    if (plain) {
        j.close(']');
        s->psi.add_component(std::make_unique<SlaterDeterminant>(std::move(blocks)));
    }

    // Padé on every group pair, a1 = 2 mu R/(2 l + d - 1) (builders/jastrow.cpp:48-63):
    // same-spin pairs of a determinant group are P-wave (l = 1), opposite spins S-wave.
    j.key("pade");
    j.open('[');
    for (std::size_t ga = 0; ga < s->groups.size(); ++ga)
        for (std::size_t gb = ga; gb < s->groups.size(); ++gb) {
            const ParticleGroup& A = s->groups[ga];
            const ParticleGroup& B = s->groups[gb];
            if (ga == gb && A.size() < 2) continue;
            const double R = ew.coulomb_cusp_residue(A, B);
            const int ell = ga == gb ? 1 : 0;
            const double a1 = 2.0 * 0.5 * R / static_cast<double>(2 * ell + 2 - 1);
            std::vector<Parameter> params{Parameter{"a1", a1, true},
                                          Parameter{"pade_0", bden, false}};
            auto pj = std::make_unique<PadeJastrow>(1, 1, A, B, params);
            pj->sum_over_images(s->cell);
#ifdef ALEA_GPU_DRIVER
            s->pade_specs.push_back({pj.get(), A, B, 1, 1});
#endif
            j.open('{');
            j.arr("ga", std::vector<double>{double(A.first), double(A.last)});
            j.arr("gb", std::vector<double>{double(B.first), double(B.last)});
            j.arr("a", std::vector<double>{a1});
            j.arr("b", std::vector<double>{bden});
            dump_pade_image_sum(j, s->cell, {a1}, {bden});
            dump_pade_opt(j, s->cell, {a1}, {bden}, {false, true});
            j.close('}');
            s->psi.add_component(std::move(pj));
        }
    j.close(']');

    // Ewald tables (numerics/ewald_breakup.h:67-103).
    const numerics::EwaldSetup& es = ew.setup();
    j.key("ewald");
    j.open('{');
    j.kv("r_cut", es.r_cut);
    dump_spline(j, "spline", es.long_range);
    j.arr("n1", es.n1);
    j.arr("n2", es.n2);
    j.arr("kx", es.kx);
    j.arr("ky", es.ky);
    j.arr("weight", es.weight);
    j.ki("n1_max", es.n1_max);
    j.ki("n2_max", es.n2_max);
    j.kv("inv_eps", 1.0);
    j.kv("self_energy", ew.self_energy());
    j.kv("background_energy", ew.background_energy());
    j.kv("v_long_zero", es.v_long_zero);
    j.kv("sr_k0", es.sr_k0);
    j.close('}');
    j.close('}');
    s->ham.add_component(std::move(ewald));
    return s;
}

// 2D Wigner crystal: Gaussian orbitals at explicit sites (a triangular lattice
// in a rectangular cell, alternate rows per spin), Drummond Jastrow (C = 3),
// Ewald.  Initial positions: sites plus Gaussian jitter.
std::unique_ptr<System> build_crystal(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "crystal";
    const int nx = static_cast<int>(geti(a, "nx", 10));
    const int ny = static_cast<int>(geti(a, "ny", 12));   // even
    const double rs = getd(a, "rs", 40.0);
    const double calpha = getd(a, "calpha", 0.1);
    const double tol = getd(a, "tol", 1e-6);
    const double alpha0 = getd(a, "alpha0", 0.0);
    const double pi = 3.14159265358979323846;
    const std::size_t N = static_cast<std::size_t>(nx * ny);
    const std::size_t nu = N / 2, nd = N - nu;
    s->dim = 2;
    s->np = N;
    const double alat = rs * std::sqrt(2.0 * pi / std::sqrt(3.0));
    const double Lx = nx * alat, Ly = ny * alat * std::sqrt(3.0) / 2.0;
    s->cell = SimulationCell(2, std::vector<double>{Lx, 0.0, 0.0, Ly});
    s->groups.push_back(make_group("up", 0, nu, -1.0, 2));
    s->groups.push_back(make_group("down", nu, nd, -1.0, 2));
    // Sites: row r, column c at ((c + (r%2)/2) a, r a sqrt3/2), shifted to the
    // centred cell; even rows carry spin up, odd rows spin down.
    std::vector<double> up_c, dn_c;
    for (int r = 0; r < ny; ++r)
        for (int c = 0; c < nx; ++c) {
            const double x = (c + 0.5 * (r % 2)) * alat - 0.5 * Lx;
            const double y = r * alat * std::sqrt(3.0) / 2.0 - 0.5 * Ly;
            auto& dst = (r % 2 == 0) ? up_c : dn_c;
            dst.push_back(x);
            dst.push_back(y);
        }
    const double alpha = calpha / (rs * rs);
    s->anchors = up_c;
    s->anchors.insert(s->anchors.end(), dn_c.begin(), dn_c.end());
    s->jitter = getd(a, "jitter", 1.0 / std::sqrt(4.0 * alpha));

    s->ham.add_component(std::make_unique<Kinetic>(s->groups));
    auto ewald = std::make_unique<EwaldTerm>(s->groups, 1.0, s->cell, tol);
    const EwaldTerm& ew = *ewald;

    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "crystal");
    j.ki("dim", 2);
    j.ki("np", static_cast<long long>(s->np));
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);
    std::vector<SlaterDeterminant::Block> blocks;
    j.key("slater");
    j.open('[');
    for (std::size_t gi = 0; gi < 2; ++gi) {
        const ParticleGroup& g = s->groups[gi];
        const std::vector<double>& cen = gi == 0 ? up_c : dn_c;
        std::vector<double> al(g.size(), alpha);
        j.open('{');
        j.ki("first", static_cast<long long>(g.first));
        j.ki("last", static_cast<long long>(g.last));
        j.ks("type", "gaussian");
        j.arr("centers", cen);
        j.arr("alphas", al);
        if (geti(a, "gauss_free", 0) != 0) j.ki("opt_alpha", 1);
        j.close('}');
        blocks.push_back({g.first, g.last,
                          std::make_unique<GaussianOrbitalSet>(2, cen, al, s->cell)});
    }
    j.close(']');
    auto slater = std::make_unique<SlaterDeterminant>(std::move(blocks));
    // gauss_free=1: each block's shared Gaussian width optimisable (the
    // config layer's opt-in; fixed by default, orbital_set.h:232-241)
    if (geti(a, "gauss_free", 0) != 0)
        for (Parameter& p : slater->parameters()) p.is_fixed = false;
    s->psi.add_component(std::move(slater));

    // Drummond: same-spin pairs (l = 1) in one item, opposite spins (l = 0) in another.
    const double Lcut = getd(a, "cutoff", 0.999 * s->cell.ws_radius());
    j.key("drummond");
    j.open('[');
    for (int item = 0; item < 2; ++item) {
        std::vector<JastrowGroupPair> pairs;
        if (item == 0) {
            pairs.push_back({s->groups[0], s->groups[0]});
            pairs.push_back({s->groups[1], s->groups[1]});
        } else {
            pairs.push_back({s->groups[0], s->groups[1]});
        }
        const double R = ew.coulomb_cusp_residue(pairs[0].a, pairs[0].b);
        const double gamma = 2.0 * 0.5 * R / static_cast<double>(2 * (item == 0 ? 1 : 0) + 1);
        // drummond_free=1: alpha_0, an alpha_2 term and L optimisable (the
        // linear method's parameters); otherwise alpha_0 and L fixed
        const bool dfree = geti(a, "drummond_free", 0) != 0;
        const double alpha2 = getd(a, "alpha2", 0.0);
        std::vector<Parameter> params{Parameter{"p0", alpha0, !dfree}};
        if (dfree) params.push_back(Parameter{"p2", alpha2, false});
        params.push_back(Parameter{"L", Lcut, !dfree, true});
        auto dj = std::make_unique<DrummondJastrow>(3, gamma, pairs, params);
        j.open('{');
        j.ki("C", 3);
        j.kv("gamma", gamma);
        j.kv("L", Lcut);
        if (dfree) j.arr("coeffs", std::vector<double>{alpha0, alpha2});
        else j.arr("coeffs", std::vector<double>{alpha0});
        if (dfree) {
            j.key("opt");
            j.open('[');
            for (int q = 0; q < 3; ++q) {
                j.open('{');
                j.ki("index", q);
                j.close('}');
            }
            j.close(']');
        }
        j.key("pairs");
        j.open('[');
        for (const auto& p : pairs)
            j.arr("", std::vector<double>{double(p.a.first), double(p.a.last),
                                          double(p.b.first), double(p.b.last)});
        j.close(']');
        j.close('}');
        s->psi.add_component(std::move(dj));
    }
    j.close(']');
    const numerics::EwaldSetup& es = ew.setup();
    j.key("ewald");
    j.open('{');
    j.kv("r_cut", es.r_cut);
    dump_spline(j, "spline", es.long_range);
    j.arr("n1", es.n1);
    j.arr("n2", es.n2);
    j.arr("kx", es.kx);
    j.arr("ky", es.ky);
    j.arr("weight", es.weight);
    j.ki("n1_max", es.n1_max);
    j.ki("n2_max", es.n2_max);
    j.kv("inv_eps", 1.0);
    j.kv("self_energy", ew.self_energy());
    j.kv("background_energy", ew.background_energy());
    j.kv("v_long_zero", es.v_long_zero);
    j.kv("sr_k0", es.sr_k0);
    j.close('}');
    j.arr("anchors", s->anchors);
    j.kv("jitter", s->jitter);
    j.close('}');
    s->ham.add_component(std::move(ewald));
    return s;
}

// Open 2D exciton: one electron, one hole, u = a1 r with a1 = -1 (the exact
// ground state, tests/configs/exciton_2d_cusp_m1.yaml), open Coulomb.
std::unique_ptr<System> build_exciton(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "exciton";
    s->dim = 2;
    s->np = 2;
    s->cell = SimulationCell(2);
    s->L_open = getd(a, "L", 1.0);
    s->groups.push_back(make_group("electron_group", 0, 1, -1.0, 2));
    s->groups.push_back(make_group("hole_group", 1, 1, 1.0, 2));
    s->ham.add_component(std::make_unique<Kinetic>(s->groups));
    s->ham.add_component(std::make_unique<CoulombTerm>(s->groups[0], s->groups[1], 1.0));
    const double a1 = 2.0 * 0.5 * (-1.0) / 1.0;
    std::vector<Parameter> params{Parameter{"a1", a1, true}};
    s->psi.add_component(
        std::make_unique<PadeJastrow>(1, 0, s->groups[0], s->groups[1], params));
    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "exciton");
    j.ki("dim", 2);
    j.ki("np", 2);
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);
    j.key("pade");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, 1});
    j.arr("gb", std::vector<double>{1, 2});
    j.arr("a", std::vector<double>{a1});
    j.arr("b", std::vector<double>{});
    j.close('}');
    j.close(']');
    j.key("coulomb");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, 1});
    j.arr("gb", std::vector<double>{1, 2});
    j.kv("coef", -1.0);
    j.close('}');
    j.close(']');
    j.kv("L_open", s->L_open);
    j.close('}');
    return s;
}

// 2D dipolar bosons (configs/dipoles_2d_gas_n256.yaml shape): n bosons of
// mass 1 in a hexagonal cell of area n π rs² (app.cpp:314-330), C/r^p at the
// minimum image plus the continuum tail (InversePowerTerm), and the
// zero-energy Jastrow with b = 2 μ C (μ = 1/2) and r_c = the Wigner-Seitz
// inradius (builders/jastrow.cpp:202-260).  Initial positions: uniform.
std::unique_ptr<System> build_dipoles(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "dipoles";
    const std::size_t n = static_cast<std::size_t>(geti(a, "n", 64));
    const double rs = getd(a, "rs", 0.03526184897173477);
    const double C = getd(a, "strength", 1.0);
    const double p = getd(a, "exponent", 3.0);
    const double rm = getd(a, "rm", 0.0459);
    const double pi = 3.14159265358979323846;
    s->dim = 2;
    s->np = n;
    const double area = static_cast<double>(n) * pi * rs * rs;
    const double L = std::sqrt(2.0 * area / std::sqrt(3.0));
    const std::vector<double> vec{L, 0.0, 0.5 * L, L * std::sqrt(3.0) / 2.0};
    s->cell = SimulationCell(2, vec);
    s->groups.push_back(make_group("dipoles", 0, n, 0.0, 2));
    s->ham.add_component(std::make_unique<Kinetic>(s->groups));
    auto ip = std::make_unique<InversePowerTerm>(s->groups[0], s->groups[0], C, p, s->cell);
    const double tail = ip->tail_energy();
    s->ham.add_component(std::move(ip));
    const double b = 2.0 * 0.5 * C;
    const double rc = s->cell.ws_radius();
    std::vector<Parameter> params{Parameter{"matching_radius", rm, true}};
    s->psi.add_component(
        std::make_unique<ZeroEnergyJastrow>(b, p, rc, s->groups[0], s->groups[0], params));
    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "dipoles");
    j.ki("dim", 2);
    j.ki("np", static_cast<long long>(n));
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);
    j.key("zero_energy");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, double(n)});
    j.arr("gb", std::vector<double>{0, double(n)});
    j.kv("b", b);
    j.kv("exponent", p);
    j.kv("matching_radius", rm);
    j.kv("cutoff", rc);
    j.close('}');
    j.close(']');
    j.key("inverse_power");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, double(n)});
    j.arr("gb", std::vector<double>{0, double(n)});
    j.kv("strength", C);
    j.kv("exponent", p);
    j.kv("tail", tail);
    j.close('}');
    j.close(']');
    j.close('}');
    return s;
}

// Real 3-D plane waves of the lowest shells of a cubic cell of side L: k = 2π n / L
// with n sorted by |n|², then lexicographically; k = 0 gives cos(0), every other
// ±n pair is represented by the n whose first nonzero component is positive and
// gives cos then sin.  The reference builds no 3-D shells
// (src/wavefunction/orbital_set.h:581-584), so this list is the harness's own;
// the device reads it from the setup dump.
void plane_waves_3d(double L, std::size_t n, std::vector<double>& k, std::vector<char>& is_sin) {
    const double pi = 3.14159265358979323846;
    std::vector<std::array<int, 4>> cand;   // |n|², n
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
        if (is_sin.size() >= n) break;
        const double kv[3] = {2 * pi * q[1] / L, 2 * pi * q[2] / L, 2 * pi * q[3] / L};
        for (int s = 0; s < (q[0] == 0 ? 1 : 2) && is_sin.size() < n; ++s) {
            k.insert(k.end(), kv, kv + 3);
            is_sin.push_back(static_cast<char>(s));
        }
    }
    if (is_sin.size() != n) throw std::runtime_error("plane_waves_3d: shell table too small");
}

// 3-D electron gas with backflow: cubic cell at density rs, one backflow
// determinant of plane waves per spin (channels as build_heg's: the own group
// with c_1 derived, the other group with c_0, c_1; C = 3; L = bf_L or half the
// cell side), Drummond Jastrows (C = 3, Kato cusps 1/2 for opposite and 1/4
// for like spins in 3-D, scaled by cusp, cutoff 0.999 R_WS), kinetic energy
// only: the reference has no 3-D Coulomb sum (src/numerics/ewald_breakup.cpp:211-213).
// bf=0 leaves plain plane-wave determinants instead.
std::unique_ptr<System> build_heg3d(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "heg3d";
    const std::size_t nu = static_cast<std::size_t>(geti(a, "nu", 27));
    const std::size_t nd = static_cast<std::size_t>(geti(a, "nd", 27));
    const double rs = getd(a, "rs", 5.0);
    const double pi = 3.14159265358979323846;
    s->dim = 3;
    s->np = nu + nd;
    const double L = rs * std::cbrt(4.0 * pi * static_cast<double>(s->np) / 3.0);
    const std::vector<double> vec{L, 0.0, 0.0, 0.0, L, 0.0, 0.0, 0.0, L};
    s->cell = SimulationCell(3, vec);
    s->groups.push_back(make_group("up", 0, nu, -1.0, 3));
    if (nd > 0) s->groups.push_back(make_group("down", nu, nd, -1.0, 3));
    s->ham.add_component(std::make_unique<Kinetic>(s->groups));

    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "heg3d");
    j.ki("dim", 3);
    j.ki("np", static_cast<long long>(s->np));
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);

    const bool backflow = geti(a, "bf", 1) != 0;
    if (backflow) {
        const double c_like = getd(a, "bf_like", 0.1);
        const double c_un0 = getd(a, "bf_un0", 0.1), c_un1 = getd(a, "bf_un1", 0.0);
        const double Lb = getd(a, "bf_L", 0.5 * L);
        j.key("backflow");
        j.open('[');
        for (std::size_t gi = 0; gi < s->groups.size(); ++gi) {
            const ParticleGroup& g = s->groups[gi];
            std::vector<double> kv;
            std::vector<char> is_sin;
            plane_waves_3d(L, g.size(), kv, is_sin);
            j.open('{');
            j.ki("first", static_cast<long long>(g.first));
            j.ki("last", static_cast<long long>(g.last));
            j.ks("type", "plane_wave");
            j.arr("k", kv);
            j.arr("is_sin", std::vector<double>(is_sin.begin(), is_sin.end()));
            std::vector<BackflowSlaterDeterminant::Channel> chans;
            j.key("channels");
            j.open('[');
            for (std::size_t hi = 0; hi < s->groups.size(); ++hi) {
                const ParticleGroup& h = s->groups[hi];
                BackflowSlaterDeterminant::Channel ch;
                ch.source_first = h.first;
                ch.source_last = h.last;
                ch.truncation = 3;
                std::vector<double> full;
                if (hi == gi) {
                    ch.params = {Parameter{"", c_like, false}, Parameter{"", Lb, true}};
                    full = {c_like, 3.0 * c_like / Lb};
                } else {
                    ch.params = {Parameter{"", c_un0, false}, Parameter{"", c_un1, false},
                                 Parameter{"", Lb, true}};
                    full = {c_un0, c_un1};
                }
                j.open('{');
                j.ki("source_first", static_cast<long long>(h.first));
                j.ki("source_last", static_cast<long long>(h.last));
                j.ki("C", 3);
                j.arr("coeffs", full);
                j.kv("L", Lb);
                j.ki("zero_slope", hi == gi ? 1 : 0);
                std::vector<double> opt;
                for (std::size_t q = 0; q < ch.params.size(); ++q)
                    if (!ch.params[q].is_fixed) opt.push_back(static_cast<double>(q));
                j.arr("opt_index", opt);
                j.close('}');
                chans.push_back(std::move(ch));
            }
            j.close(']');
            j.close('}');
            std::vector<BackflowSlaterDeterminant::Block> bb;
            bb.push_back({g.first, g.last, std::make_unique<PlaneWaveOrbitalSet>(3, kv, is_sin)});
            s->psi.add_component(std::make_unique<BackflowSlaterDeterminant>(
                std::move(bb), std::move(chans), s->cell));
        }
        j.close(']');
    } else {
        std::vector<SlaterDeterminant::Block> blocks;
        j.key("slater");
        j.open('[');
        for (const ParticleGroup& g : s->groups) {
            std::vector<double> kv;
            std::vector<char> is_sin;
            plane_waves_3d(L, g.size(), kv, is_sin);
            j.open('{');
            j.ki("first", static_cast<long long>(g.first));
            j.ki("last", static_cast<long long>(g.last));
            j.ks("type", "plane_wave");
            j.arr("k", kv);
            j.arr("is_sin", std::vector<double>(is_sin.begin(), is_sin.end()));
            j.close('}');
            blocks.push_back({g.first, g.last, std::make_unique<PlaneWaveOrbitalSet>(3, kv, is_sin)});
        }
        j.close(']');
        s->psi.add_component(std::make_unique<SlaterDeterminant>(std::move(blocks)));
    }

    const double alpha0 = getd(a, "alpha0", 0.0);
    if (geti(a, "jastrow", 1) != 0 && nd > 0) {
        const double Lcut = getd(a, "cutoff", 0.999 * s->cell.ws_radius());
        j.key("drummond");
        j.open('[');
        for (int item = 0; item < 2; ++item) {
            std::vector<JastrowGroupPair> pairs;
            if (item == 0) {
                pairs.push_back({s->groups[0], s->groups[0]});
                pairs.push_back({s->groups[1], s->groups[1]});
            } else {
                pairs.push_back({s->groups[0], s->groups[1]});
            }
            // 2 μ R / (2l + d - 1) with μ = 1/2, R = 1, d = 3; cusp=0 gives a smooth
            // Jastrow (the kinetic-only Hamiltonian then has no 1/r local energy)
            const double gamma = getd(a, "cusp", 1.0) / static_cast<double>(2 * (item == 0 ? 1 : 0) + 2);
            std::vector<Parameter> params{Parameter{"p0", alpha0, true}, Parameter{"L", Lcut, true, true}};
            auto dj = std::make_unique<DrummondJastrow>(3, gamma, pairs, params);
            j.open('{');
            j.ki("C", 3);
            j.kv("gamma", gamma);
            j.kv("L", Lcut);
            j.arr("coeffs", std::vector<double>{alpha0});
            j.key("pairs");
            j.open('[');
            for (const auto& p : pairs)
                j.arr("", std::vector<double>{double(p.a.first), double(p.a.last),
                                              double(p.b.first), double(p.b.last)});
            j.close(']');
            j.close('}');
            s->psi.add_component(std::move(dj));
        }
        j.close(']');
    }
    j.close('}');
    return s;
}

// Open 3-D cell, the shape of the reference's own 3-D backflow test
// (tests/test_backflow_slater.cpp:198-214): three like-spin particles [0, 3)
// in Gaussian orbitals of one shared width, displaced by each other (zero
// slope, c_0 = 0.2, c_2 = -0.04, L = 2.4) and by two holes [3, 5) (c_0 =
// -0.12, c_1 = 0.08, c_2 = 0.03, L = 2.8); a Padé Jastrow a r/(1 + b r)
// between the particles and the holes; kinetic energy and the open Coulomb
// attraction between the two groups.  Initial positions uniform in [-L/2, L/2)³.
std::unique_ptr<System> build_gauss3d(const Args& a) {
    auto s = std::make_unique<System>();
    s->kind = "gauss3d";
    s->dim = 3;
    s->np = 5;
    s->cell = SimulationCell(3);
    s->L_open = getd(a, "L", 2.0);
    s->groups.push_back(make_group("particles", 0, 3, -1.0, 3));
    s->groups.push_back(make_group("holes", 3, 2, 1.0, 3));
    s->ham.add_component(std::make_unique<Kinetic>(s->groups));
    s->ham.add_component(std::make_unique<CoulombTerm>(s->groups[0], s->groups[1], 1.0));
    const std::vector<double> centers{-0.9, 0.1, 0.2, 0.8, 0.3, -0.4, 0.1, -0.8, 0.6};
    const std::vector<double> alphas{0.5, 0.5, 0.5};
    Json& j = s->setup;
    j.open('{');
    j.ks("kind", "gauss3d");
    j.ki("dim", 3);
    j.ki("np", 5);
    dump_cell(j, s->cell);
    dump_groups(j, s->groups);
    const double c0 = 0.2, L1 = 2.4;
    std::vector<BackflowSlaterDeterminant::Channel> chans(2);
    chans[0].source_first = 0;
    chans[0].source_last = 3;
    chans[0].truncation = 3;
    chans[0].params = {Parameter{"", c0, false}, Parameter{"", -0.04, false}, Parameter{"", L1, true}};
    chans[1].source_first = 3;
    chans[1].source_last = 5;
    chans[1].truncation = 3;
    chans[1].params = {Parameter{"", -0.12, false}, Parameter{"", 0.08, false}, Parameter{"", 0.03, false},
                       Parameter{"", 2.8, true}};
    j.key("backflow");
    j.open('[');
    j.open('{');
    j.ki("first", 0);
    j.ki("last", 3);
    j.ks("type", "gaussian");
    j.arr("centers", centers);
    j.arr("alphas", alphas);
    j.key("channels");
    j.open('[');
    const std::vector<std::vector<double>> full{{c0, 3.0 * c0 / L1, -0.04}, {-0.12, 0.08, 0.03}};
    const double Ls[2] = {L1, 2.8};
    for (int q = 0; q < 2; ++q) {
        j.open('{');
        j.ki("source_first", static_cast<long long>(chans[q].source_first));
        j.ki("source_last", static_cast<long long>(chans[q].source_last));
        j.ki("C", 3);
        j.arr("coeffs", full[q]);
        j.kv("L", Ls[q]);
        j.ki("zero_slope", q == 0 ? 1 : 0);
        j.close('}');
    }
    j.close(']');
    j.close('}');
    j.close(']');
    std::vector<BackflowSlaterDeterminant::Block> bb;
    bb.push_back({0, 3, std::make_unique<GaussianOrbitalSet>(3, centers, alphas)});
    s->psi.add_component(std::make_unique<BackflowSlaterDeterminant>(std::move(bb), std::move(chans), s->cell));
    const double pa = getd(a, "pade_a", -0.3), pb = getd(a, "pade_b", 0.5);
    std::vector<Parameter> params{Parameter{"a1", pa, true}, Parameter{"pade_0", pb, true}};
    s->psi.add_component(std::make_unique<PadeJastrow>(1, 1, s->groups[0], s->groups[1], params));
    j.key("pade");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, 3});
    j.arr("gb", std::vector<double>{3, 5});
    j.arr("a", std::vector<double>{pa});
    j.arr("b", std::vector<double>{pb});
    j.close('}');
    j.close(']');
    j.key("coulomb");
    j.open('[');
    j.open('{');
    j.arr("ga", std::vector<double>{0, 3});
    j.arr("gb", std::vector<double>{3, 5});
    j.kv("coef", -1.0);
    j.close('}');
    j.close(']');
    j.kv("L_open", s->L_open);
    j.close('}');
    return s;
}

std::unique_ptr<System> build_system(const Args& a) {
    const std::string k = gets(a, "system", "heg");
    if (k == "heg") return build_heg(a);
    if (k == "heg3d") return build_heg3d(a);
    if (k == "gauss3d") return build_gauss3d(a);
    if (k == "crystal") return build_crystal(a);
    if (k == "exciton") return build_exciton(a);
    if (k == "dipoles") return build_dipoles(a);
    throw std::runtime_error("unknown system " + k);
}

// Initial positions with the reference App's semantics (app.cpp:56-112):
// numerics::Random (mt19937_64) in walker, particle, dimension order; uniform
// fractional coordinates in [-1/2, 1/2) mapped through the cell vectors,
// uniform in [-L/2, L/2) for an open cell, or anchor + jitter * N(0, 1).
void initialize(WalkerEnsemble& ens, const System& s, std::uint64_t seed) {
    numerics::Random rng(seed);
    const std::size_t np = s.np, dim = s.dim;
    const auto av = s.cell.vectors();
    std::vector<double> pos(np * dim);
    for (Walker& w : ens.walkers()) {
        for (std::size_t p = 0; p < np; ++p) {
            if (!s.anchors.empty()) {
                for (std::size_t d = 0; d < dim; ++d)
                    pos[p * dim + d] = s.anchors[p * dim + d] + s.jitter * rng.gaussian();
            } else if (s.cell.is_periodic()) {
                double f[3];
                for (std::size_t i = 0; i < dim; ++i) f[i] = rng.uniform(-0.5, 0.5);
                for (std::size_t d = 0; d < dim; ++d) {
                    double acc = 0.0;
                    for (std::size_t i = 0; i < dim; ++i) acc += f[i] * av[i * dim + d];
                    pos[p * dim + d] = acc;
                }
            } else {
                for (std::size_t d = 0; d < dim; ++d)
                    pos[p * dim + d] = rng.uniform(-0.5 * s.L_open, 0.5 * s.L_open);
            }
        }
        w.set_positions(pos);
    }
}

void put_positions(Json& j, const std::string& k, const WalkerEnsemble& ens) {
    j.key(k);
    j.open('[');
    for (const Walker& w : ens.walkers()) j.arr("", w.positions());
    j.close(']');
}

// Array with no key (the writer's "arr" with an empty key writes `"":`); used
// inside lists, so strip that.
std::string fix_empty_keys(std::string s) {
    std::string out;
    out.reserve(s.size());
    for (std::size_t i = 0; i < s.size(); ++i) {
        if (s.compare(i, 3, "\"\":") == 0) {
            i += 2;
            continue;
        }
        out += s[i];
    }
    return out;
}

// The estimators named by the arguments, built as the reference's estimator
// builders do: gofr (gofr_rmax, gofr_bins), density (dens_rmax, dens_bins,
// dens_pp = one series per particle) and sofk (sofk_kmax).
std::vector<std::unique_ptr<Estimator>> make_estimators(const Args& a, const System& s) {
    std::vector<std::unique_ptr<Estimator>> e;
    const std::span<const ParticleGroup> groups(s.groups);
    if (geti(a, "gofr_bins", 0) > 0)
        e.push_back(std::make_unique<PairCorrelation>(groups, s.dim, getd(a, "gofr_rmax", 1.0),
                                                      static_cast<int>(geti(a, "gofr_bins", 0)), s.cell));
    if (geti(a, "dens_bins", 0) > 0)
        e.push_back(std::make_unique<Density>(groups, s.dim, getd(a, "dens_rmax", 1.0),
                                              static_cast<int>(geti(a, "dens_bins", 0)),
                                              geti(a, "dens_pp", 0) != 0, s.cell));
    if (getd(a, "sofk_kmax", 0.0) > 0.0)
        e.push_back(std::make_unique<StructureFactor>(groups, s.cell, getd(a, "sofk_kmax", 0.0)));
    return e;
}

// Every series and scalar of a run result, under "estimators".
void put_results(Json& j, const RunResult& r) {
    j.key("estimators");
    j.open('{');
    for (const auto& [k, v] : r.series) j.arr(k, v);
    for (const auto& [k, v] : r.scalars) j.kv(k, v);
    j.close('}');
}

int run(const std::string& mode, const Args& a) {
    auto sys = build_system(a);
    const std::size_t nw = static_cast<std::size_t>(geti(a, "nw", 4));
    const std::uint64_t seed = static_cast<std::uint64_t>(geti(a, "seed", 12345));
    const std::uint64_t init_seed = static_cast<std::uint64_t>(geti(a, "init_seed", seed));

    if (mode == "setup") {
        std::printf("%s\n", fix_empty_keys(sys->setup.s).c_str());
        return 0;
    }
    WalkerEnsemble ens(nw, sys->groups, sys->dim, sys->cell);
    initialize(ens, *sys, init_seed);
    // pos_file=PATH: the walkers' positions instead, whitespace-separated AoS [w][p][d]
    if (const std::string pf = gets(a, "pos_file", ""); !pf.empty()) {
        std::FILE* f = std::fopen(pf.c_str(), "r");
        if (!f) throw std::runtime_error("cannot open " + pf);
        std::vector<double> pos(sys->np * sys->dim);
        for (Walker& w : ens.walkers()) {
            for (double& x : pos)
                if (std::fscanf(f, "%lf", &x) != 1) throw std::runtime_error("short pos_file " + pf);
            w.set_positions(pos);
        }
        std::fclose(f);
    }

    Json out;
    out.open('{');
    out.ks("mode", mode);
    if (mode == "init") {
        put_positions(out, "positions", ens);
    } else if (mode == "eval") {
        WalkerSet ws(nw, sys->np, sys->dim, sys->cell);
        for (Walker& w : ens.walkers()) ws.add_walker(w);
        ws.load_all();
        TrialWavefunction psi = sys->psi.clone();
        Hamiltonian ham = sys->ham.clone();
        psi.evaluate_batch(ws);
        ham.evaluate_batch(ws);
        put_positions(out, "positions", ens);
        out.arr("log_psi", ws.log_psi());
        out.arr("local_energy", ws.local_energies());
        out.arr("grad", ws.gradients());
        out.arr("lap", ws.laplacians());
        if (ws.has_phase()) {
            out.arr("phase_grad", ws.phase_gradients());
            out.arr("phase_lap", ws.phase_laplacians());
            out.arr("local_energy_imag", ws.local_energies_imag());
        }
        out.key("component_log_psi");
        out.open('[');
        for (const auto& c : psi.components()) out.arr("", c->log_psi_c());
        out.close(']');
        // d ln psi_c / d p_k of every component's optimisable parameters
        out.key("param_derivs");
        out.open('[');
        for (const auto& c : psi.components()) {
            std::vector<double> d(c->num_optimizable_params() * nw);
            if (!d.empty()) c->compute_parameter_derivatives(ws, d);
            out.arr("", d);
        }
        out.close(']');
        // d(grad_d ln psi_c)/d p_k and d(lap_d ln psi_c)/d p_k, [n_opt][np*dim*nw]
        // per component (empty when the component does not supply them)
        out.key("param_grad_derivs");
        out.open('[');
        for (const auto& c : psi.components()) {
            const std::size_t n = c->num_optimizable_params() * sys->np * sys->dim * nw;
            std::vector<double> dg(n), dl(n);
            const bool ok = n > 0 && c->supports_parameter_gradient_derivatives() &&
                            c->compute_parameter_gradient_derivatives(ws, dg, dl);
            out.open('{');
            out.ki("ok", ok ? 1 : 0);
            out.arr("grad", ok ? dg : std::vector<double>{});
            out.arr("lap", ok ? dl : std::vector<double>{});
            out.close('}');
        }
        out.close(']');
        // Kinetic alone, to separate the potential.
        Hamiltonian kin;
        kin.add_component(std::make_unique<Kinetic>(sys->groups));
        kin.evaluate_batch(ws);
        out.arr("kinetic", ws.local_energies());
    } else if (mode == "vmc") {
        VMCConfig c;
        c.n_equilibration_blocks = static_cast<int>(geti(a, "eq", 0));
        c.n_accumulation_blocks = static_cast<int>(geti(a, "acc", 2));
        c.n_steps = static_cast<int>(geti(a, "steps", 3));
        c.n_substeps = static_cast<int>(geti(a, "substeps", 1));
        c.tau = getd(a, "tau", 1.0);
        c.use_drift = geti(a, "drift", 0) != 0;
        c.n_threads = static_cast<int>(geti(a, "threads", static_cast<long long>(nw)));
        c.seed = seed;
        const int T = std::min<int>(c.n_threads, static_cast<int>(nw));
        put_positions(out, "initial_positions", ens);
        VMC vmc(c, ens, sys->psi, sys->ham);
        std::vector<std::vector<double>> el(static_cast<std::size_t>(T));
        vmc.set_measure_hook([&](const WalkerSet& ws, const TrialWavefunction&) {
            auto& v = el[static_cast<std::size_t>(omp_get_thread_num())];
            for (double e : ws.local_energies()) v.push_back(e);
        });
        auto ests = make_estimators(a, *sys);
        const bool with_ests = !ests.empty();
        if (with_ests) vmc.set_estimators(std::move(ests));
        vmc.run();
        if (with_ests) put_results(out, vmc.run_result());
        out.kv("energy", vmc.energy());
        out.kv("energy_error", vmc.energy_error());
        out.kv("variance", vmc.energy_variance());
        out.kv("acceptance", vmc.acceptance_ratio());
        out.ki("threads", T);
        out.key("thread_local_energy");
        out.open('[');
        for (const auto& v : el) out.arr("", v);
        out.close(']');
        out.arr("final_positions", vmc.final_configurations());
        out.arr("block_energies", vmc.block_energies());
    } else if (mode == "dmc" || mode == "bench") {
        const bool bench = mode == "bench";
        const std::string method = gets(a, "method", "dmc");
        const int host_threads = omp_get_max_threads();
        if (bench && method == "vmc") {
            VMCConfig c;
            c.n_equilibration_blocks = 0;
            c.n_accumulation_blocks = 1;
            c.n_steps = static_cast<int>(geti(a, "steps", 2));
            c.n_substeps = 1;
            c.tau = getd(a, "tau", 1.0);
            c.n_threads = static_cast<int>(geti(a, "threads", host_threads));
            c.seed = seed;
            VMC vmc(c, ens, sys->psi, sys->ham);
            std::vector<double> stamps;
            vmc.set_measure_hook([&](const WalkerSet&, const TrialWavefunction&) {
                if (omp_get_thread_num() == 0)
                    stamps.push_back(std::chrono::duration<double>(
                        std::chrono::steady_clock::now().time_since_epoch()).count());
            });
            vmc.run();
            out.ki("threads", c.n_threads);
            out.arr("stamps", stamps);
            out.kv("acceptance", vmc.acceptance_ratio());
        } else {
            DMCConfig c;
            c.n_equilibration_blocks = static_cast<int>(geti(a, "eq", 0));
            c.n_accumulation_blocks = static_cast<int>(geti(a, "acc", 1));
            c.n_steps = static_cast<int>(geti(a, "steps", 3));
            c.n_substeps = static_cast<int>(geti(a, "substeps", 1));
            c.tau = getd(a, "tau", 0.5);
            c.n_threads = static_cast<int>(
                geti(a, "threads", bench ? host_threads : static_cast<long long>(nw)));
            c.seed = seed;
            c.population_generations = getd(a, "generations", 10.0);
            // forward walking: fw_lags=t0,t1,... (imaginary times), fw_interval
            const std::string fw = gets(a, "fw_lags", "");
            for (std::size_t p0 = 0; p0 < fw.size();) {
                const std::size_t p1 = std::min(fw.find(',', p0), fw.size());
                c.forward_walking_lags.push_back(std::stod(fw.substr(p0, p1 - p0)));
                p0 = p1 + 1;
            }
            c.forward_walking_interval = static_cast<std::size_t>(geti(a, "fw_interval", 1));
            if (!bench) put_positions(out, "initial_positions", ens);
            DMC dmc(c, ens, sys->psi, sys->ham);
            // ckpt=1: the milestone checkpoint hook's calls (DMC::run's eq /
            // a25 / a50 / a75 snapshots): tag, blocks done, SoA positions
            Json ck;
            ck.open('[');
            if (geti(a, "ckpt", 0) != 0)
                dmc.set_checkpoint_hook([&ck](const WalkerSet& ws, std::string_view tag, int done) {
                    ck.open('{');
                    ck.ks("tag", std::string(tag));
                    ck.ki("blocks_done", done);
                    ck.ki("nw", static_cast<long long>(ws.num_walkers()));
                    ck.arr("positions", ws.positions());
                    ck.close('}');
                });
            if (!c.forward_walking_lags.empty()) {
                // each lag: the same estimators, labelled fw<i> as the builders do
                std::vector<std::vector<std::unique_ptr<Estimator>>> per_lag(c.forward_walking_lags.size());
                for (std::size_t i = 0; i < per_lag.size(); ++i) {
                    per_lag[i] = make_estimators(a, *sys);
                    for (auto& e : per_lag[i]) e->set_output_label("fw" + std::to_string(i));
                }
                dmc.set_forward_walking_estimators(std::move(per_lag));
            }
            std::vector<double> stamps, wsum, ewsum, nws;
            std::vector<std::vector<double>> el, wt, ids;
            dmc.set_measure_hook([&](const WalkerSet& ws, const TrialWavefunction&) {
                stamps.push_back(std::chrono::duration<double>(
                    std::chrono::steady_clock::now().time_since_epoch()).count());
                nws.push_back(static_cast<double>(ws.num_walkers()));
                double sw = 0.0, se = 0.0;
                for (std::size_t w = 0; w < ws.num_walkers(); ++w) {
                    sw += ws.weights()[w];
                    se += ws.weights()[w] * ws.local_energies()[w];
                }
                wsum.push_back(sw);
                ewsum.push_back(se);
                if (!bench) {
                    el.emplace_back(ws.local_energies().begin(), ws.local_energies().end());
                    wt.emplace_back(ws.weights().begin(), ws.weights().end());
                    ids.emplace_back(ws.ids().begin(), ws.ids().end());
                }
            });
            auto ests = make_estimators(a, *sys);
            const bool with_ests = !ests.empty();
            if (with_ests) dmc.set_estimators(std::move(ests));
            const auto t0 = std::chrono::steady_clock::now();
            dmc.run();
            const double wall =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (with_ests || !c.forward_walking_lags.empty()) put_results(out, dmc.run_result());
            ck.close(']');
            if (geti(a, "ckpt", 0) != 0) {
                out.key("checkpoints");
                out.s += ck.s;
                out.first = false;
            }
            out.ki("threads", c.n_threads);
            out.kv("wall", wall);
            out.arr("stamps", stamps);
            out.arr("walkers", nws);
            out.arr("weight_sum", wsum);
            out.arr("weighted_energy_sum", ewsum);
            out.ks("summary_first_line", "");
            if (!bench) {
                out.key("local_energy");
                out.open('[');
                for (const auto& v : el) out.arr("", v);
                out.close(']');
                out.key("weights");
                out.open('[');
                for (const auto& v : wt) out.arr("", v);
                out.close(']');
                out.key("ids");
                out.open('[');
                for (const auto& v : ids) out.arr("", v);
                out.close(']');
                out.arr("final_positions", dmc.final_configurations());
            }
        }
    } else if (mode == "chain") {
        // VMC, then DMC seeded from VMC's final configurations the way
        // carry_over_walkers / seed_walker_rows do it (app.cpp:1068-1098):
        // a fresh ensemble of dmc_nw walkers, walker w on row w mod rows.
        VMCConfig vc;
        vc.n_equilibration_blocks = static_cast<int>(geti(a, "eq", 0));
        vc.n_accumulation_blocks = static_cast<int>(geti(a, "acc", 1));
        vc.n_steps = static_cast<int>(geti(a, "steps", 2));
        vc.n_substeps = static_cast<int>(geti(a, "substeps", 1));
        vc.tau = getd(a, "tau", 1.0);
        vc.n_threads = static_cast<int>(nw);
        vc.seed = seed;
        put_positions(out, "initial_positions", ens);
        VMC vmc(vc, ens, sys->psi, sys->ham);
        vmc.run();
        const std::vector<double> rows = vmc.final_configurations();
        out.arr("vmc_final_positions", rows);
        const std::size_t nw2 = static_cast<std::size_t>(geti(a, "dmc_nw", static_cast<long long>(nw)));
        const std::size_t row = sys->np * sys->dim, n_rows = rows.size() / row;
        WalkerEnsemble ens2(nw2, sys->groups, sys->dim, sys->cell);
        {
            std::size_t w = 0;
            for (Walker& wk : ens2.walkers()) {
                wk.set_positions(std::span<const double>(rows).subspan((w % n_rows) * row, row));
                ++w;
            }
        }
        DMCConfig dc;
        dc.n_equilibration_blocks = static_cast<int>(geti(a, "dmc_eq", 0));
        dc.n_accumulation_blocks = static_cast<int>(geti(a, "dmc_acc", 1));
        dc.n_steps = static_cast<int>(geti(a, "dmc_steps", 3));
        dc.n_substeps = 1;
        dc.tau = getd(a, "dmc_tau", 0.5);
        dc.n_threads = static_cast<int>(nw2);
        dc.seed = static_cast<std::uint64_t>(geti(a, "dmc_seed", static_cast<long long>(seed) + 1));
        dc.population_generations = getd(a, "generations", 10.0);
        DMC dmc(dc, ens2, sys->psi, sys->ham);
        std::vector<double> wsum, ewsum, nws;
        dmc.set_measure_hook([&](const WalkerSet& ws, const TrialWavefunction&) {
            nws.push_back(static_cast<double>(ws.num_walkers()));
            double sw = 0.0, se = 0.0;
            for (std::size_t w = 0; w < ws.num_walkers(); ++w) {
                sw += ws.weights()[w];
                se += ws.weights()[w] * ws.local_energies()[w];
            }
            wsum.push_back(sw);
            ewsum.push_back(se);
        });
        dmc.run();
        out.arr("walkers", nws);
        out.arr("weight_sum", wsum);
        out.arr("weighted_energy_sum", ewsum);
        out.arr("final_positions", dmc.final_configurations());
#ifdef ALEA_GPU_DRIVER
    } else if (mode == "gpu_pair") {
        const std::string method = gets(a, "method", "dmc");
        const gpu::PackedSystem packed = gpu::pack_system(ens, sys->psi, sys->ham, sys->pade_specs);
        WalkerEnsemble ens_gpu = ens;
        put_positions(out, "initial_positions", ens);
        const int threads = static_cast<int>(geti(a, "threads", static_cast<long long>(nw)));
        if (method == "vmc") {
            VMCConfig c;
            c.n_equilibration_blocks = static_cast<int>(geti(a, "eq", 0));
            c.n_accumulation_blocks = static_cast<int>(geti(a, "acc", 2));
            c.n_steps = static_cast<int>(geti(a, "steps", 3));
            c.n_substeps = static_cast<int>(geti(a, "substeps", 1));
            c.tau = getd(a, "tau", 1.0);
            c.n_threads = threads;
            c.seed = seed;
            VMC ref(c, ens, sys->psi, sys->ham);
            ref.run();
            gpu::GpuVMC dev(c, ens_gpu, packed);
            dev.run();
            out.arr("ref_block_energies", ref.block_energies());
            out.arr("gpu_block_energies", dev.block_energies());
            out.kv("ref_energy", ref.energy());
            out.kv("gpu_energy", dev.energy());
            out.kv("ref_acceptance", ref.acceptance_ratio());
            out.kv("gpu_acceptance", dev.acceptance_ratio());
            out.arr("ref_final_positions", ref.final_configurations());
            out.arr("gpu_final_positions", dev.final_configurations());
            out.ks("gpu_summary", dev.summary());
        } else {
            DMCConfig c;
            c.n_equilibration_blocks = static_cast<int>(geti(a, "eq", 0));
            c.n_accumulation_blocks = static_cast<int>(geti(a, "acc", 1));
            c.n_steps = static_cast<int>(geti(a, "steps", 3));
            c.n_substeps = static_cast<int>(geti(a, "substeps", 1));
            c.tau = getd(a, "tau", 0.5);
            c.n_threads = threads;
            c.seed = seed;
            c.population_generations = getd(a, "generations", 10.0);
            DMC ref(c, ens, sys->psi, sys->ham);
            ref.run();
            gpu::GpuDMC dev(c, ens_gpu, packed);
            dev.run();
            out.arr("ref_block_energies", ref.block_energies());
            out.arr("gpu_block_energies", dev.block_energies());
            out.kv("ref_energy", ref.energy());
            out.kv("gpu_energy", dev.energy());
            out.kv("ref_energy_error", ref.energy_error());
            out.kv("gpu_energy_error", dev.energy_error());
            out.arr("ref_final_positions", ref.final_configurations());
            out.arr("gpu_final_positions", dev.final_configurations());
            out.ks("gpu_summary", dev.summary());
            const RunResult rr = dev.run_result();
            out.ks("gpu_method", rr.method);
            out.ki("gpu_result_scalars", static_cast<long long>(rr.scalars.size()));
        }
#endif
    } else if (mode == "estimate") {
        // acc blocks of `steps` configurations each: configuration (b, s) is a
        // fresh App initialisation from init_seed + 1000 b + s, walker w
        // weighted by 0.25 + 0.125 ((5w + 3s + b) mod 13).
        const int n_blocks = static_cast<int>(geti(a, "acc", 2));
        const int n_steps = static_cast<int>(geti(a, "steps", 3));
        auto ests = make_estimators(a, *sys);
        out.key("configurations");
        out.open('[');
        for (int b = 0; b < n_blocks; ++b) {
            for (auto& e : ests) e->start_block();
            for (int st = 0; st < n_steps; ++st) {
                WalkerEnsemble e2(nw, sys->groups, sys->dim, sys->cell);
                initialize(e2, *sys, init_seed + 1000 * static_cast<std::uint64_t>(b) +
                                         static_cast<std::uint64_t>(st));
                WalkerSet ws(nw, sys->np, sys->dim, sys->cell);
                for (Walker& w : e2.walkers()) ws.add_walker(w);
                ws.load_all();
                std::vector<double> wt(nw);
                for (std::size_t w = 0; w < nw; ++w)
                    wt[w] = 0.25 + 0.125 * static_cast<double>((5 * w + 3 * st + b) % 13);
                for (auto& e : ests) e->accumulate(ws, wt);
                out.open('{');
                out.arr("positions", ws.positions());
                out.arr("weights", wt);
                out.close('}');
            }
            for (auto& e : ests) e->stop_block();
        }
        out.close(']');
        RunResult rr;
        for (auto& e : ests) e->write_results(rr);
        put_results(out, rr);
    } else {
        throw std::runtime_error("unknown mode " + mode);
    }
    out.close('}');
    std::printf("%s\n", fix_empty_keys(out.s).c_str());
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness MODE key=value...\n");
        return 2;
    }
    Args a;
    for (int i = 2; i < argc; ++i) {
        const std::string s = argv[i];
        const auto eq = s.find('=');
        if (eq == std::string::npos) {
            std::fprintf(stderr, "bad argument %s\n", s.c_str());
            return 2;
        }
        a[s.substr(0, eq)] = s.substr(eq + 1);
    }
    try {
        return run(argv[1], a);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_harness: %s\n", e.what());
        return 1;
    }
}
