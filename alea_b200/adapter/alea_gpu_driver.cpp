// GpuVMC / GpuDMC and pack_system: see alea_gpu_driver.h.
#include "alea_gpu_driver.h"

#include <chrono>
#include <cmath>
#include <sstream>
#include <stdexcept>

#include "hamiltonian/ewald_term.h"
#include "hamiltonian/kinetic.h"
#include "numerics/long_range_breakup.h"
#include "numerics/pair_radial.h"
#include "wavefunction/orbital_set.h"
#include "wavefunction/pade_jastrow.h"
#include "wavefunction/slater_determinant.h"

namespace alea::gpu {

const double* PackedSystem::keep(std::vector<double> v) {
    d_.push_back(std::move(v));
    return d_.back().data();
}

const int* PackedSystem::keepi(std::vector<int> v) {
    i_.push_back(std::move(v));
    return i_.back().data();
}

namespace {

void set_spline(alea_gpu_spline& out, const numerics::LongRangeSpline& sp, const double* scaled) {
    out.r_cut = sp.r_cut;
    out.inv_delta = sp.inv_delta;
    out.n_knots = sp.n_knots;
    out.scaled = scaled;
}

int rank_of(const ParticleGroup& g) { return static_cast<int>(g.first); }

}  // namespace

PackedSystem pack_system(const WalkerEnsemble& ens, const TrialWavefunction& psi, const Hamiltonian& ham,
                         const std::vector<PadeTermSpec>& pade) {
    PackedSystem P;
    alea_gpu_system& y = P.sys_;
    const SimulationCell& cell = ens.cell();
    const std::size_t dim = ens.dim();
    if (dim != 2) throw std::invalid_argument("pack_system: the device path is two-dimensional");
    y.dim = 2;
    y.n_particles = static_cast<int>(ens.n_particles());
    y.periodic = cell.is_periodic() ? 1 : 0;
    if (y.periodic) {
        const auto v = cell.vectors();
        for (std::size_t i = 0; i < 4; ++i) y.lattice[i] = v[i];
    }
    const auto groups = ens.groups();
    if (groups.size() > ALEA_GPU_MAX_GROUPS) throw std::invalid_argument("pack_system: too many groups");
    for (const ParticleGroup& g : groups) {
        alea_gpu_group& o = y.groups[y.n_groups++];
        o.first = static_cast<int>(g.first);
        o.last = static_cast<int>(g.last);
        o.charge = g.charge;
        for (std::size_t d = 0; d < dim && d < g.inv_mass.size(); ++d) o.inv_mass[d] = g.inv_mass[d];
    }

    for (const auto& comp : psi.components()) {
        const WavefunctionComponent* c = comp.get();
        if (dynamic_cast<const SlaterDeterminant*>(c)) {
            for (const NodalBlockView& b : c->nodal_blocks()) {
                const auto* pw = dynamic_cast<const PlaneWaveOrbitalSet*>(b.orbitals);
                if (!pw)
                    throw std::invalid_argument("pack_system: only plane-wave Slater blocks are flattened");
                if (y.n_blocks == ALEA_GPU_MAX_BLOCKS) throw std::invalid_argument("pack_system: too many blocks");
                const std::size_t n = pw->size();
                // a sine vanishes at the origin, a cosine is 1 there
                std::vector<double> origin(dim, 0.0), val(n), grad(n * dim), lap(n * dim);
                pw->evaluate(origin, dim, val, grad, lap, 0, 1);
                std::vector<int> is_sin(n);
                for (std::size_t i = 0; i < n; ++i) is_sin[i] = std::abs(val[i]) < 0.5 ? 1 : 0;
                const auto k = pw->kvectors();
                alea_gpu_orbitals& o = y.blocks[y.n_blocks++];
                o.first = static_cast<int>(b.first);
                o.last = static_cast<int>(b.last);
                o.type = ALEA_ORB_PLANE_WAVE;
                o.k = P.keep(std::vector<double>(k.begin(), k.begin() + n * dim));
                o.is_sin = P.keepi(std::move(is_sin));
            }
            continue;
        }
        if (const auto* pj = dynamic_cast<const PadeJastrow*>(c)) {
            const PadeTermSpec* spec = nullptr;
            for (const PadeTermSpec& s : pade)
                if (s.term == c) spec = &s;
            if (!spec) throw std::invalid_argument("pack_system: a Padé Jastrow without its group spec");
            if (y.n_terms == ALEA_GPU_MAX_TERMS) throw std::invalid_argument("pack_system: too many pair terms");
            const auto prm = pj->parameters();
            const std::size_t N = static_cast<std::size_t>(spec->num_order);
            const std::size_t M = static_cast<std::size_t>(spec->den_order);
            if (prm.size() != N + M || N + M > 16) throw std::invalid_argument("pack_system: Padé orders");
            std::vector<double> a, b;
            for (std::size_t i = 0; i < N; ++i) a.push_back(prm[i].value);
            for (std::size_t i = 0; i < M; ++i) b.push_back(prm[N + i].value);
            alea_gpu_pair_term& T = y.terms[y.n_terms++];
            T.kind = ALEA_PAIR_PADE;
            T.n_pairs = 1;
            const ParticleGroup& A = rank_of(spec->group_a) <= rank_of(spec->group_b) ? spec->group_a : spec->group_b;
            const ParticleGroup& B = &A == &spec->group_a ? spec->group_b : spec->group_a;
            T.pairs[0][0] = static_cast<int>(A.first);
            T.pairs[0][1] = static_cast<int>(A.last);
            T.pairs[0][2] = static_cast<int>(B.first);
            T.pairs[0][3] = static_cast<int>(B.last);
            T.num_order = static_cast<int>(N);
            T.den_order = static_cast<int>(M);
            for (std::size_t i = 0; i < N + M; ++i) T.coeffs[i] = prm[i].value;
            if (pj->sums_over_images()) {
                // the breakup PeriodicPairSum builds for u - u_inf
                const double rc = cell.ws_radius();
                numerics::BreakupOptions opt{};
                opt.k_continuum = 20.0 * 3.14159265358979323846 / rc;
                opt.k_max = 300.0 / rc;
                opt.n_continuum = 150;
                opt.k_cut = 5.0 * std::min(std::hypot(cell.reciprocal()[0], cell.reciprocal()[1]),
                                           std::hypot(cell.reciprocal()[2], cell.reciprocal()[3]));
                const numerics::LongRangeBreakup br =
                    numerics::build_long_range_breakup(cell, numerics::pade_radial(a, b, rc), opt);
                T.image_sum = 1;
                set_spline(T.short_range, br.spline(), P.keep(br.spline().scaled));
                T.u_inf = numerics::pade_limit(a, b);
                T.kset.n_k = static_cast<int>(br.weight().size());
                T.kset.n1 = P.keepi(std::vector<int>(br.n1().begin(), br.n1().end()));
                T.kset.n2 = P.keepi(std::vector<int>(br.n2().begin(), br.n2().end()));
                T.kset.kx = P.keep(std::vector<double>(br.kx().begin(), br.kx().end()));
                T.kset.ky = P.keep(std::vector<double>(br.ky().begin(), br.ky().end()));
                T.kset.weight = P.keep(std::vector<double>(br.weight().begin(), br.weight().end()));
            }
            continue;
        }
        throw std::invalid_argument("pack_system: no device form of the wavefunction component '" + c->name() +
                                    "'");
    }

    for (const auto& comp : ham.components()) {
        const HamiltonianComponent* h = comp.get();
        if (dynamic_cast<const Kinetic*>(h)) continue;
        if (const auto* ew = dynamic_cast<const EwaldTerm*>(h)) {
            const numerics::EwaldSetup& es = ew->setup();
            y.ewald.enabled = 1;
            y.ewald.r_cut = es.r_cut;
            set_spline(y.ewald.long_range, es.long_range, P.keep(es.long_range.scaled));
            // the last knot holds f_l(r_c) = f(r_c) = 1/(ε r_c)
            const int nk = es.long_range.n_knots;
            y.ewald.inv_eps = es.long_range.scaled[3 * (nk - 1)] * es.long_range.r_cut;
            y.ewald.constant = ew->self_energy() + ew->background_energy();
            y.ewald.kset.n_k = static_cast<int>(es.weight.size());
            y.ewald.kset.n1 = P.keepi(es.n1);
            y.ewald.kset.n2 = P.keepi(es.n2);
            y.ewald.kset.kx = P.keep(es.kx);
            y.ewald.kset.ky = P.keep(es.ky);
            y.ewald.kset.weight = P.keep(es.weight);
            continue;
        }
        throw std::invalid_argument("pack_system: no device form of the Hamiltonian term '" + h->name() + "'");
    }
    return P;
}

// ───────────────────────── drivers ───────────────────────────────────────

GpuDriverBase::GpuDriverBase(WalkerEnsemble& ensemble, const PackedSystem& sys, int device)
    : ens_(ensemble), sys_(sys), device_(device) {
    initial_ = soa_positions();
}

GpuDriverBase::~GpuDriverBase() {
    if (ctx_) alea_gpu_destroy(ctx_);
}

std::vector<double> GpuDriverBase::soa_positions() const {
    const std::size_t nw = ens_.num_walkers(), np = ens_.n_particles(), dim = ens_.dim();
    std::vector<double> soa(nw * np * dim);
    std::size_t w = 0;
    for (const Walker& wk : ens_.walkers()) {
        const auto p = wk.positions();
        for (std::size_t i = 0; i < np; ++i)
            for (std::size_t d = 0; d < dim; ++d) soa[(i * dim + d) * nw + w] = p[i * dim + d];
        ++w;
    }
    return soa;
}

void GpuDriverBase::reload_configurations() { initial_ = soa_positions(); }

void GpuDriverBase::check(int rc, const char* what) const {
    if (rc == ALEA_OK) return;
    const std::string msg = std::string("gpu driver: ") + what + ": " + alea_gpu_last_error(ctx_);
    if (rc == ALEA_ERR_INVALID || rc == ALEA_ERR_UNSUPPORTED) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

void GpuDriverBase::open(int capacity) {
    if (ctx_) alea_gpu_destroy(ctx_);
    ctx_ = nullptr;
    check(alea_gpu_create(sys_.get(), device_, capacity, &ctx_), "alea_gpu_create");
    check(alea_gpu_upload_walkers(ctx_, initial_.data(), static_cast<int>(ens_.num_walkers())),
          "alea_gpu_upload_walkers");
}

std::vector<double> GpuDriverBase::final_configurations() const {
    if (!ctx_) return {};
    int nw = 0;
    check(alea_gpu_final_configurations(ctx_, nullptr, &nw), "alea_gpu_final_configurations");
    std::vector<double> rows(static_cast<std::size_t>(nw) * ens_.n_particles() * ens_.dim());
    check(alea_gpu_final_configurations(ctx_, rows.data(), &nw), "alea_gpu_final_configurations");
    return rows;
}

namespace {

alea_gpu_run_config run_config(int n_eq, int n_acc, int n_steps, int n_sub, double tau, bool drift,
                               int n_threads, std::uint64_t seed) {
    alea_gpu_run_config rc{};
    rc.n_equilibration_blocks = n_eq;
    rc.n_accumulation_blocks = n_acc;
    rc.n_steps = n_steps;
    rc.n_substeps = n_sub;
    rc.tau = tau;
    rc.use_drift = drift ? 1 : 0;
    rc.n_streams = n_threads;
    rc.seed = seed;
    return rc;
}

void common_scalars(RunResult& r, const alea_gpu_run_result& res) {
    r.add_scalar("energy", res.energy);
    r.add_scalar("energy_error", res.energy_error);
    r.add_scalar("energy_variance", res.variance);
    r.add_scalar("acceptance_ratio", res.acceptance);
    r.add_scalar("walltime_s", res.walltime_s);
}

}  // namespace

GpuVMC::GpuVMC(const VMCConfig& cfg, WalkerEnsemble& ensemble, const PackedSystem& sys, int device)
    : GpuDriverBase(ensemble, sys, device), cfg_(cfg) {}

// VMC::run (src/qmc/vmc.cpp:189-431): the threads' streams become the
// device's random streams over contiguous walker ranges, one chain each.
void GpuVMC::run() {
    const int nw = static_cast<int>(ens_.num_walkers());
    open(nw);
    const alea_gpu_run_config rc = run_config(cfg_.n_equilibration_blocks, cfg_.n_accumulation_blocks,
                                              cfg_.n_steps, cfg_.n_substeps, cfg_.tau, cfg_.use_drift,
                                              cfg_.n_threads, cfg_.seed);
    const int chains = std::min(cfg_.n_threads, nw);
    blocks_.assign(static_cast<std::size_t>(chains) * cfg_.n_accumulation_blocks, 0.0);
    check(alea_gpu_vmc_run(ctx_, &rc, &res_, blocks_.data()), "alea_gpu_vmc_run");
}

std::string GpuVMC::summary() const {
    std::stringstream ss;
    ss << "vmc: E = " << res_.energy << " +/- " << res_.energy_error << "  var = " << res_.variance
       << "  acc = " << res_.acceptance;
    return ss.str();
}

RunResult GpuVMC::run_result() const {
    RunResult r;
    r.method = "vmc";
    common_scalars(r, res_);
    r.add_scalar("tau", cfg_.tau);
    r.add_scalar("n_walkers", static_cast<double>(ens_.num_walkers()));
    r.add_scalar("n_threads", static_cast<double>(cfg_.n_threads));
    r.add_scalar("n_equilibration_blocks", static_cast<double>(cfg_.n_equilibration_blocks));
    r.add_scalar("n_accumulation_blocks", static_cast<double>(cfg_.n_accumulation_blocks));
    r.add_scalar("n_steps", static_cast<double>(cfg_.n_steps));
    r.add_scalar("n_substeps", static_cast<double>(cfg_.n_substeps));
    r.add_metadata("device", "gpu");
    r.add_series("block_energy", blocks_);
    r.check_unique_keys();
    return r;
}

GpuDMC::GpuDMC(const DMCConfig& cfg, WalkerEnsemble& ensemble, const PackedSystem& sys, int device)
    : GpuDriverBase(ensemble, sys, device), cfg_(cfg) {
    if (cfg.reweighting != Reweighting::bare || cfg.branch_cutoff != BranchCutoff::universal)
        throw std::invalid_argument("gpu dmc: the device runs bare reweighting with the universal cutoff");
    if (!cfg.forward_walking_lags.empty())
        throw std::invalid_argument("gpu dmc: forward walking goes through alea_gpu_set_forward_walking");
}

// DMC::run (src/qmc/dmc.cpp:525-884): crowds of the population as the
// device's streams, branching on the serial stream, population control
// toward the ensemble's target.
void GpuDMC::run() {
    const int target = static_cast<int>(ens_.target_walkers());
    open(std::max(2 * target + 2, static_cast<int>(ens_.num_walkers())));
    alea_gpu_run_config rc = run_config(cfg_.n_equilibration_blocks, cfg_.n_accumulation_blocks, cfg_.n_steps,
                                        cfg_.n_substeps, cfg_.tau, true, cfg_.n_threads, cfg_.seed);
    rc.target_walkers = target;
    rc.population_generations = cfg_.population_generations;
    rc.branch_cutoff_alpha = cfg_.branch_cutoff_alpha;
    blocks_.assign(static_cast<std::size_t>(cfg_.n_accumulation_blocks), 0.0);
    check(alea_gpu_dmc_run(ctx_, &rc, &res_, blocks_.data()), "alea_gpu_dmc_run");
}

std::string GpuDMC::summary() const {
    std::stringstream ss;
    ss << "dmc: E = " << res_.energy << " +/- " << res_.energy_error << "  var = " << res_.variance
       << "  acc = " << res_.acceptance;
    return ss.str();
}

RunResult GpuDMC::run_result() const {
    RunResult r;
    r.method = "dmc";
    common_scalars(r, res_);
    r.add_scalar("etrial_final", res_.e_trial);
    r.add_scalar("tau", cfg_.tau);
    r.add_scalar("n_walkers", static_cast<double>(ens_.target_walkers()));
    r.add_scalar("n_threads", static_cast<double>(cfg_.n_threads));
    r.add_scalar("n_equilibration_blocks", static_cast<double>(cfg_.n_equilibration_blocks));
    r.add_scalar("n_accumulation_blocks", static_cast<double>(cfg_.n_accumulation_blocks));
    r.add_scalar("n_steps", static_cast<double>(cfg_.n_steps));
    r.add_scalar("n_substeps", static_cast<double>(cfg_.n_substeps));
    r.add_scalar("population_generations", cfg_.population_generations);
    r.add_scalar("branch_cutoff_alpha", cfg_.branch_cutoff_alpha);
    r.add_scalar("final_population", static_cast<double>(res_.n_walkers));
    r.add_metadata("device", "gpu");
    r.add_series("block_energy", blocks_);
    r.check_unique_keys();
    return r;
}

}  // namespace alea::gpu
