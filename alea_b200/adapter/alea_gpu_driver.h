// Reference-side drop-in for the walker path: VMC and DMC drivers of the
// reference's Driver interface (src/qmc/driver.h:20-60) that run on the B200
// through the C ABI of include/alea_gpu.h, and pack_system, which flattens a
// reference-built trial function and Hamiltonian into the ABI's
// alea_gpu_system.
//
// This file is compiled against the reference's own headers (it is the code
// a maintainer adds beside src/qmc/vmc.h and src/qmc/dmc.h); the App selects
// these drivers where a stage says `device: gpu` (src/io/parser.cpp:113-116,
// src/qmc/app.cpp:873, :920).  oracle/Makefile builds it with the reference's
// hot-path sources into oracle/_ref/ref_harness_gpu.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "../../include/alea_gpu.h"
#include "hamiltonian/hamiltonian.h"
#include "population/particle_group.h"
#include "population/walker_ensemble.h"
#include "qmc/dmc.h"
#include "qmc/driver.h"
#include "qmc/vmc.h"
#include "wavefunction/trial_wavefunction.h"

namespace alea::gpu {

// What a reference component does not tell about itself through its public
// interface: the particle groups a Padé Jastrow couples and its numerator and
// denominator orders (the App's Jastrow builder knows them when it builds the
// term, src/builders/jastrow.cpp).  One entry per PadeJastrow component.
struct PadeTermSpec {
    const WavefunctionComponent* term = nullptr;
    ParticleGroup group_a, group_b;
    int num_order = 1, den_order = 1;
};

// An alea_gpu_system and the tables it points into.
class PackedSystem {
public:
    const alea_gpu_system* get() const noexcept { return &sys_; }

private:
    friend PackedSystem pack_system(const WalkerEnsemble&, const TrialWavefunction&, const Hamiltonian&,
                                    const std::vector<PadeTermSpec>&);
    alea_gpu_system sys_{};
    std::vector<std::vector<double>> d_;
    std::vector<std::vector<int>> i_;
    const double* keep(std::vector<double> v);
    const int* keepi(std::vector<int> v);
};

// The flat description of ψ and H for the device:
//   cell and groups        from the ensemble (WalkerEnsemble::cell/groups)
//   plane-wave blocks      SlaterDeterminant::nodal_blocks -> PlaneWaveOrbitalSet:
//                          kvectors(), and sine/cosine from the orbital's value
//                          at the origin (0 for a sine)
//   Padé Jastrows          parameters() with the spec's groups and orders; an
//                          image-summed term (sums_over_images) is split with
//                          the reference's own breakup on PeriodicPairSum's
//                          options (src/wavefunction/periodic_pair_sum.cpp:21-60)
//   Ewald                  EwaldTerm::setup(), self_energy(), background_energy();
//                          1/ε from the long-range spline's last knot (f_l = 1/(ε r_c))
//   kinetic                nothing (the device always adds it)
// Anything else throws std::invalid_argument, naming the component: the
// caller keeps the CPU driver for that system.
PackedSystem pack_system(const WalkerEnsemble& ens, const TrialWavefunction& psi, const Hamiltonian& ham,
                         const std::vector<PadeTermSpec>& pade);

// Common part of the two drivers: one device context for the run's
// population, created in run() and kept for final_configurations().
class GpuDriverBase : public Driver {
public:
    GpuDriverBase(WalkerEnsemble& ensemble, const PackedSystem& sys, int device);
    ~GpuDriverBase() override;
    GpuDriverBase(const GpuDriverBase&) = delete;
    GpuDriverBase& operator=(const GpuDriverBase&) = delete;

    [[nodiscard]] std::vector<double> final_configurations() const override;
    void reload_configurations() override;

    double energy() const noexcept { return res_.energy; }
    double energy_error() const noexcept { return res_.energy_error; }
    double energy_variance() const noexcept { return res_.variance; }
    double acceptance_ratio() const noexcept { return res_.acceptance; }
    const std::vector<double>& block_energies() const noexcept { return blocks_; }

protected:
    // the ensemble's walkers as the ABI's SoA planes [p*dim*nw + d*nw + w]
    std::vector<double> soa_positions() const;
    void check(int rc, const char* what) const;
    void open(int capacity);

    WalkerEnsemble& ens_;
    const PackedSystem& sys_;
    int device_;
    alea_gpu_ctx* ctx_ = nullptr;
    std::vector<double> initial_;          // SoA positions read at construction / reload
    alea_gpu_run_result res_{};
    std::vector<double> blocks_;
};

class GpuVMC final : public GpuDriverBase {
public:
    GpuVMC(const VMCConfig& cfg, WalkerEnsemble& ensemble, const PackedSystem& sys, int device = 0);
    void run() override;
    [[nodiscard]] std::string summary() const override;
    [[nodiscard]] RunResult run_result() const override;

private:
    VMCConfig cfg_;
};

class GpuDMC final : public GpuDriverBase {
public:
    GpuDMC(const DMCConfig& cfg, WalkerEnsemble& ensemble, const PackedSystem& sys, int device = 0);
    void run() override;
    [[nodiscard]] std::string summary() const override;
    [[nodiscard]] RunResult run_result() const override;

private:
    DMCConfig cfg_;
};

}  // namespace alea::gpu
