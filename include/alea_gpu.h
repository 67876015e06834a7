/*
 * alea_gpu.h — C ABI of the B200 walker hot path (VMC/DMC) for Alea.
 *
 * A host that already builds Alea's trial wavefunction and Hamiltonian (the
 * reference's builders, or this library's own host setup) describes the
 * system once with a flat alea_gpu_system, creates a context on a device, and
 * then drives walkers that stay resident in HBM.  Plain C types only; every
 * function returns ALEA_OK (0) or an ALEA_ERR_* code, and
 * alea_gpu_last_error() returns the context's last message.
 *
 * Reference interfaces these entry points replace (paths in ItaloAlb/alea):
 *   alea_gpu_create / destroy      the per-thread ψ/H clones and WalkerSet of
 *                                  src/qmc/vmc.cpp:23-62, src/qmc/dmc.cpp:69-163
 *   alea_gpu_upload_walkers        WalkerSet::load_all (src/population/walker_set.cpp:54-70)
 *   alea_gpu_evaluate              TrialWavefunction::evaluate_batch
 *                                  (src/wavefunction/trial_wavefunction.cpp:19-35) +
 *                                  Hamiltonian::evaluate_batch (src/hamiltonian/hamiltonian.cpp:18-29)
 *   alea_gpu_download_walkers      WalkerSet positions/log_psi/gradients/laplacians/
 *                                  local_energies/weights (src/population/walker_set.h:86-152)
 *   alea_gpu_move                  ParticleBatch::propose_move_batch + TrialWavefunction::
 *                                  ratio_batch + apply_move_batch_deferred + WalkerSet::apply_move
 *                                  (src/population/particle_batch.cpp:43-57,
 *                                  src/wavefunction/trial_wavefunction.cpp:46-91,
 *                                  src/population/walker_set.cpp:72-107)
 *   alea_gpu_vmc_step              VMC::run_step (src/qmc/vmc.cpp:157-187), per-thread streams
 *                                  of VMC::VMC (src/qmc/vmc.cpp:45-61)
 *   alea_gpu_dmc_advance           DMC::advance_measure over the crowds of DMC::run_one_step
 *                                  (src/qmc/dmc.cpp:339-419, :693-702)
 *   alea_gpu_dmc_branch            WalkerSet::branch + TrialWavefunction::permute_caches
 *                                  (src/population/walker_set.cpp:187-239, src/qmc/dmc.cpp:733-734)
 *   alea_gpu_vmc_run / dmc_run     VMC::run / DMC::run (src/qmc/vmc.cpp:189-431,
 *                                  src/qmc/dmc.cpp:525-884)
 *
 * Layouts follow the reference's WalkerSet: positions, gradients and
 * Laplacians are SoA with the walker index fastest, [p*dim*nw + d*nw + w].
 */
#ifndef ALEA_GPU_H
#define ALEA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALEA_GPU_ABI_VERSION 2

enum {
    ALEA_OK = 0,
    ALEA_ERR_INVALID = 1,      /* bad argument or system description */
    ALEA_ERR_CUDA = 2,         /* a CUDA call failed */
    ALEA_ERR_UNSUPPORTED = 3,  /* valid, but outside what the kernels implement */
    ALEA_ERR_SINGULAR = 4,     /* a determinant became singular or nonfinite */
    ALEA_ERR_TIMEOUT = 5,      /* a bounded device wait ran out */
    ALEA_ERR_NOMEM = 6,        /* device allocation failed / capacity exceeded */
    ALEA_ERR_CANCELLED = 7     /* a served job was cancelled (alea_gpu_cancel) */
};

enum { ALEA_ORB_PLANE_WAVE = 0, ALEA_ORB_GAUSSIAN = 1, ALEA_ORB_TWISTED_PLANE_WAVE = 2 };
enum { ALEA_PAIR_PADE = 0, ALEA_PAIR_DRUMMOND = 1, ALEA_PAIR_ZERO_ENERGY = 2 };

#define ALEA_GPU_MAX_GROUPS 8
#define ALEA_GPU_MAX_BLOCKS 4
#define ALEA_GPU_MAX_TERMS 8
#define ALEA_GPU_MAX_PAIRS 4
#define ALEA_GPU_MAX_COULOMB 8
#define ALEA_GPU_MAX_OPT 4

/* Quintic-Hermite long-range spline of the optimized breakup
 * (src/numerics/long_range_spline.h:41-48): 3 coefficients per knot, scaled
 * by delta^alpha. */
typedef struct {
    double r_cut;
    double inv_delta;
    int n_knots;
    const double* scaled; /* [3 * n_knots] */
} alea_gpu_spline;

/* Half-space reciprocal vectors k = n1 b1 + n2 b2 (+ n3 b3 in 3-D) with their
 * weights (src/numerics/ewald_breakup.h:73-77).  n3 and kz are read only in
 * a 3-D system (NULL otherwise). */
typedef struct {
    int n_k;
    const int* n1;
    const int* n2;
    const double* kx;
    const double* ky;
    const double* weight;
    const int* n3;
    const double* kz;
} alea_gpu_kset;

typedef struct {
    int first, last;      /* particle index range [first, last) */
    double charge;
    double inv_mass[3];   /* per dimension */
} alea_gpu_group;

/* One determinant block (src/wavefunction/slater_determinant.h:60-64).
 * Twisted plane waves e^{i(k+θ)·r} (src/wavefunction/complex_orbital_set.h:78-182)
 * make the determinant complex (ComplexSlaterDeterminant,
 * src/wavefunction/complex_slater_determinant.h:20-104); then every block is
 * twisted and DMC runs fixed phase. */
typedef struct {
    int first, last;
    int type;                 /* ALEA_ORB_* */
    const double* k;          /* plane waves: [n * dim]; twisted: q = k + θ [n * dim] */
    const int* is_sin;        /* plane waves: [n], nonzero = sine */
    const double* centers;    /* Gaussians: [n * dim] */
    const double* alphas;     /* Gaussians: [n] */
    int opt_alpha;            /* Gaussians of one shared width: that width is an optimisable
                                 parameter (GaussianOrbitalSet, src/wavefunction/orbital_set.h:226-286) */
} alea_gpu_orbitals;

/* A pair Jastrow: Padé u = Σ a_k r^k / (1 + Σ b_k r^k) on one group pair,
 * optionally summed over periodic images (short-range spline + k-space
 * weights), or Drummond-Towler-Needs on one or more group pairs. */
typedef struct {
    int kind;                               /* ALEA_PAIR_* */
    int n_pairs;
    int pairs[ALEA_GPU_MAX_PAIRS][4];       /* a_first, a_last, b_first, b_last */
    int num_order, den_order;               /* Padé */
    double coeffs[16];                      /* Padé [a_1..a_N, b_1..b_M] */
    int image_sum;                          /* Padé in a periodic cell with Ewald */
    alea_gpu_spline short_range;            /* f_long of u - u_inf, subtracted inside r_cut */
    double u_inf;
    alea_gpu_kset kset;                     /* reciprocal half of the image sum */
    int C;                                  /* Drummond truncation order */
    double gamma, L;                        /* Drummond cusp and cutoff */
    int n_coeffs;
    double dcoeffs[16];                     /* Drummond [alpha_0, alpha_2..alpha_N] */
    /* zero-energy pair function on one group pair
       (src/wavefunction/zero_energy_jastrow.h:16-55): C1 K0(kappa r^-s) inside
       the matching radius, C2 exp(-C3/r - C3/(2 r_c - r)) up to the cutoff */
    double ze_b;                            /* 2 mu C of the pair's C/r^p core */
    double ze_exponent;                     /* p > 2 */
    double ze_matching_radius, ze_cutoff;
    /* The term's optimisable parameters, in the order of its Parameter list
       (the linear method's, WavefunctionComponent::compute_parameter_derivatives,
       src/wavefunction/wavefunction_component.h:165-171).  opt_index: Padé, the
       index into coeffs (a_1..a_N, then b_1..b_M); Drummond, 0 = alpha_0,
       i = alpha_{i+1} for 1 <= i < n_coeffs, n_coeffs = the cutoff L.  An
       image-summed Padé also carries, per parameter, the breakup of
       du/dp - its r -> infinity limit on the term's k set
       (src/wavefunction/pade_jastrow.cpp:208-248). */
    int n_opt;
    int opt_index[ALEA_GPU_MAX_OPT];
    double opt_inf[ALEA_GPU_MAX_OPT];
    alea_gpu_spline opt_short_range[ALEA_GPU_MAX_OPT];
    const double* opt_weight[ALEA_GPU_MAX_OPT];   /* [kset.n_k] */
} alea_gpu_pair_term;

/* 2-D Ewald sum of the Coulomb interaction (src/hamiltonian/ewald_term.h). */
typedef struct {
    int enabled;
    double r_cut;
    double inv_eps;
    double constant;              /* self + background energy */
    alea_gpu_spline long_range;
    alea_gpu_kset kset;
} alea_gpu_ewald;

/* Open-boundary Coulomb between two groups (src/hamiltonian/coulomb.h). */
typedef struct {
    int a_first, a_last, b_first, b_last;
    double coef;                  /* q_a q_b / epsilon */
} alea_gpu_coulomb;

/* C / r^p between two groups at the minimum image, plus the continuum tail
 * of the images outside the Wigner-Seitz cell (src/hamiltonian/inverse_power.h). */
typedef struct {
    int a_first, a_last, b_first, b_last;
    double strength, exponent;
    double tail;                  /* constant added to every configuration */
} alea_gpu_inverse_power;

/* One backflow channel: the particles [source_first, source_last) displace
 * every row of the determinant by η(r) r, η = (1 - r/L)^C Σ_k c_k r^k for
 * r < L (src/wavefunction/backflow_function.h:11-37; coeffs are c_0..c_N with
 * a like-spin channel's c_1 = C c_0 / L already filled in).
 * zero_slope marks that derived c_1; n_opt / opt_index name the channel's
 * optimisable parameters in BackflowFunction's order [c_0, (c_1 unless
 * zero_slope), c_2.., L] (backflow_function.h:111-135), ascending. */
typedef struct {
    int source_first, source_last;
    int C;
    double L;
    int n_coeffs;
    double coeffs[16];
    int zero_slope;
    int n_opt;
    int opt_index[ALEA_GPU_MAX_OPT];
} alea_gpu_backflow_channel;

/* A backflow Slater determinant over the rows [first, last) of one spin group
 * (src/wavefunction/backflow_slater_determinant.h:15-80): orbitals (plane
 * waves or Gaussians, as alea_gpu_orbitals) at the quasi-coordinates
 * x_i = r_i + Σ_c Σ_j η_c(r_ij) r_ij.  A system with backflow determinants
 * has no plain determinant blocks. */
typedef struct {
    int first, last;
    int type;                 /* ALEA_ORB_PLANE_WAVE or ALEA_ORB_GAUSSIAN */
    const double* k;
    const int* is_sin;
    const double* centers;
    const double* alphas;
    int n_channels;
    alea_gpu_backflow_channel channels[4];
} alea_gpu_backflow;

typedef struct {
    int dim;                      /* 2, or 3: orthorhombic or open cells, backflow or plain
                                     determinants, Drummond / minimum-image Padé terms,
                                     3-D Ewald (kset.kz), open Coulomb */
    int n_particles;
    int periodic;
    double lattice[9];            /* reduced lattice vectors, row-major [i*dim + d]
                                     (SimulationCell::vectors()) */
    int n_groups;
    alea_gpu_group groups[ALEA_GPU_MAX_GROUPS];
    int n_blocks;
    alea_gpu_orbitals blocks[ALEA_GPU_MAX_BLOCKS];
    int n_terms;
    alea_gpu_pair_term terms[ALEA_GPU_MAX_TERMS];
    alea_gpu_ewald ewald;
    int n_coulomb;
    alea_gpu_coulomb coulomb[ALEA_GPU_MAX_COULOMB];
    int n_inverse_power;
    alea_gpu_inverse_power inverse_power[ALEA_GPU_MAX_COULOMB];
    int n_backflow;
    alea_gpu_backflow backflow[2];
} alea_gpu_system;

typedef struct alea_gpu_ctx alea_gpu_ctx;

/* Create a context for `sys` on CUDA device `device` with room for
 * `capacity` walkers.  Copies every table; `sys` may be freed afterwards. */
int alea_gpu_create(const alea_gpu_system* sys, int device, int capacity, alea_gpu_ctx** out);
int alea_gpu_destroy(alea_gpu_ctx* ctx);
/* Last error message of the context (or of the last failed create when ctx
 * is NULL).  Valid until the next call on the context. */
const char* alea_gpu_last_error(const alea_gpu_ctx* ctx);
int alea_gpu_abi_version(void);

/* Positions of nw walkers, SoA [p*dim*nw + d*nw + w]; they are wrapped into
 * the cell and fully evaluated (ψ, derivatives, E_L).  Weights reset to 1.
 * ALEA_ERR_INVALID for a nonfinite position (nothing is launched);
 * ALEA_ERR_SINGULAR when a walker's determinant is singular (coincident
 * same-spin particles, say), as the reference's evaluation throws
 * (src/wavefunction/slater_determinant.cpp:927-928). */
int alea_gpu_upload_walkers(alea_gpu_ctx* ctx, const double* positions, int nw);
int alea_gpu_evaluate(alea_gpu_ctx* ctx);
int alea_gpu_num_walkers(const alea_gpu_ctx* ctx, int* nw);
/* Copies of the committed walker state; any pointer may be NULL.
 * gradients/laplacians are the totals ∇ln ψ and ∂²_d ln ψ, SoA like positions. */
int alea_gpu_download_walkers(alea_gpu_ctx* ctx, double* positions, double* log_psi,
                              double* gradients, double* laplacians, double* local_energy,
                              double* weights);
/* Phase part of ∇ln ψ and ∂²_d ln ψ (SoA like positions) and Im E_L per
 * walker, for a complex (twisted) determinant: the phase planes of WalkerSet
 * (src/population/walker_set.h:104-131) and the imaginary local energy of
 * Kinetic::add_phase_terms (src/hamiltonian/kinetic.cpp:75-99).  Any pointer
 * may be NULL; ALEA_ERR_INVALID for a real trial function. */
int alea_gpu_download_phase(alea_gpu_ctx* ctx, double* phase_gradients, double* phase_laplacians,
                            double* local_energy_imag);

/* One single-particle move of particle p for every walker: propose
 * new_pos [d*nw + w], compute log|ψ'/ψ|, its phase (π on a node crossing),
 * ∇ln ψ and ∂²_d ln ψ of p at the proposed position, then commit the walkers
 * with accept[w] != 0 (accept may be NULL: ratio only).  Outputs may be NULL. */
int alea_gpu_move(alea_gpu_ctx* ctx, int p, const double* new_pos, const uint8_t* accept,
                  double* log_ratio, double* phase, double* new_grad, double* new_lap);
/* Refresh every derivative and recompute E_L (before reading them after moves). */
int alea_gpu_measure(alea_gpu_ctx* ctx);
/* The same move in the reference's three steps (ParticleBatch::
 * propose_move_batch, src/population/particle_batch.cpp:43-57;
 * WavefunctionComponent::ratio_batch and the masked commit,
 * src/wavefunction/wavefunction_component.h:82-110): propose keeps particle
 * p's new positions [d*nw + w]; ratio returns what alea_gpu_move returns for
 * them; commit applies them to the walkers with mask[w] != 0 and drops the
 * proposal.  ALEA_ERR_INVALID when ratio/commit name another particle than
 * the pending proposal. */
int alea_gpu_propose(alea_gpu_ctx* ctx, int p, const double* new_pos);
int alea_gpu_ratio(alea_gpu_ctx* ctx, int p, double* log_ratio, double* phase, double* new_grad, double* new_lap);
int alea_gpu_commit(alea_gpu_ctx* ctx, int p, const uint8_t* mask);
/* Refresh and E_L of every walker into el [nw] (Hamiltonian::evaluate_batch
 * after TrialWavefunction::refresh_derivatives). */
int alea_gpu_local_energy(alea_gpu_ctx* ctx, double* el);

/* Random streams: stream t starts from xoshiro256++ seeded with
 * stream_seed(seed, kind, t) (src/numerics/random.h:52-56). */
#define ALEA_STREAM_VMC 0x766d632d74687264ULL   /* "vmc-thrd" */
#define ALEA_STREAM_DMC 0x646d632d74687264ULL   /* "dmc-thrd" */
#define ALEA_STREAM_BRANCH 0x646d632d62726368ULL /* "dmc-brch" */
int alea_gpu_set_streams(alea_gpu_ctx* ctx, uint64_t seed, uint64_t kind, int n_streams);
/* The same, under the name of the fused-driver contract. */
int alea_gpu_set_rng_streams(alea_gpu_ctx* ctx, uint64_t stage_seed, uint64_t stream_kind, int n_streams);

typedef struct {
    double tau;
    int n_substeps;
    int use_drift;       /* Langevin (1) or symmetric Metropolis (0) */
} alea_gpu_vmc_params;

typedef struct {
    double energy_sum;       /* Σ_w E_L (VMC) or Σ_w weight·E_L (DMC) */
    double energy_sq_sum;
    double weight_sum;       /* DMC: Σ_w weight */
    int64_t n_accepted;
    int64_t n_proposed;
    int64_t n_cut;           /* DMC: walker sweeps tapered by the branch cutoff */
    int n_walkers;           /* walkers at the end of the step */
} alea_gpu_step_stats;

/* One VMC step: n_substeps sweeps, then the derivative refresh and E_L.  The
 * walkers are split over the streams in contiguous even ranges, as VMC's
 * threads are (src/qmc/vmc.cpp:45-61). */
int alea_gpu_vmc_step(alea_gpu_ctx* ctx, const alea_gpu_vmc_params* prm, alea_gpu_step_stats* out);
/* n_steps VMC steps, statistics summed over the steps (n_walkers: the last). */
int alea_gpu_vmc_steps(alea_gpu_ctx* ctx, const alea_gpu_vmc_params* prm, int n_steps, alea_gpu_step_stats* out);

/* The same VMC step as alea_gpu_vmc_step, allocating nothing (no counterpart
 * in the reference).  For callers that must not allocate device memory once
 * a run is set up: a serving loop that admits jobs by their HBM footprint
 * has reserved that memory at admission, and alea_gpu_vmc_step's scratch
 * grows with cudaFree + cudaMalloc (a cudaMalloc that can then fail mid-run,
 * a cudaFree that synchronizes the whole device under the other jobs).
 *   - Scratch: the sweep's random numbers and the step's reduced statistics
 *     live in one file-scope static device array of ALEA_GPU_NOALLOC_RANDOMS
 *     + 32 doubles (8 MiB + 256 B).  A step needs n_substeps × n_particles ×
 *     3 × walkers doubles of it; a larger step returns ALEA_ERR_INVALID with a
 *     message and launches nothing.
 *   - Set-up: the first call on a context looks up the array's device
 *     address (cudaGetSymbolAddress, with the context's device current);
 *     make that first call before any stream capture.
 *   - Sharing: the array exists once per device and every context on that
 *     device uses it, so calls that overlap on the GPU race.  It keeps the
 *     last call's contents; each call writes all the scratch it reads before
 *     reading it, so nothing in it needs to start at zero.
 *   - alea_gpu_set_streams must have been called (that call may allocate).
 * Results equal alea_gpu_vmc_step's: same kernels, same random numbers;
 * the energy sums are reduced on the device (rounding order differs).
 * alea_gpu_last_kernel_ms reports the step's sweep, as after a VMC step. */
#define ALEA_GPU_NOALLOC_RANDOMS 1048576
int alea_gpu_vmc_step_noalloc(alea_gpu_ctx* ctx, const alea_gpu_vmc_params* prm, alea_gpu_step_stats* out);

typedef struct {
    double tau;
    int n_substeps;
    double e_trial, e_ref;          /* PopulationControl state before the step */
    double e_cut, e_max;            /* branch-weight cutoff window */
} alea_gpu_dmc_params;

/* One DMC advance (no branching): every crowd sweeps its walkers n_substeps
 * times with drift-diffusion moves, refreshes, evaluates E_L and multiplies
 * the weights by each sweep's branch factor.  Crowds are the contiguous
 * ranges of min(n_streams, nw) even splits of the current population. */
int alea_gpu_dmc_advance(alea_gpu_ctx* ctx, const alea_gpu_dmc_params* prm, alea_gpu_step_stats* out);
/* Branch on the serial stream state[4] (xoshiro256++, advanced in place):
 * multiplicities floor(w + U), clipping to [target/5 + 1, 2 target + 1],
 * walker state gathered, weights reset to 1. */
int alea_gpu_dmc_branch(alea_gpu_ctx* ctx, uint64_t* state, int target);
/* n_steps DMC steps (advance, then branch on `branch_state`) at the fixed
 * population-control state of prm; the caller updates E_T between calls as
 * PopulationControl::update does (src/qmc/population_control.cpp:56-103), or
 * runs alea_gpu_dmc_run, which does.  Statistics summed over the steps. */
int alea_gpu_dmc_steps(alea_gpu_ctx* ctx, const alea_gpu_dmc_params* prm, int n_steps, uint64_t* branch_state,
                       int target, alea_gpu_step_stats* out);

typedef struct {
    int n_equilibration_blocks, n_accumulation_blocks, n_steps, n_substeps;
    double tau;
    int use_drift;
    int n_streams;
    uint64_t seed;
    /* DMC only */
    int target_walkers;
    double population_generations;
    double branch_cutoff_alpha;
} alea_gpu_run_config;

typedef struct {
    double energy, energy_error, variance, acceptance;
    double walltime_s;
    int n_walkers;
    double e_trial;
    int64_t n_moves;         /* single-particle moves proposed, all blocks */
    int64_t n_evaluations;   /* local energies evaluated, all blocks */
} alea_gpu_run_result;

/* Whole VMC / DMC runs, the reference drivers' loops with device sweeps.
 * block_energies (nullable) receives one mean per accumulation block (VMC:
 * one per block and stream chain, stream-major).  The context's estimators
 * (alea_gpu_add_estimator) start afresh and measure every accumulation step:
 * VMC with one chain per random stream and unit weights (vmc.cpp:331-350),
 * DMC on the whole population with the DMC weights before the branch
 * (dmc.cpp:704-706, :792-801). */
int alea_gpu_vmc_run(alea_gpu_ctx* ctx, const alea_gpu_run_config* cfg, alea_gpu_run_result* res,
                     double* block_energies);
int alea_gpu_dmc_run(alea_gpu_ctx* ctx, const alea_gpu_run_config* cfg, alea_gpu_run_result* res,
                     double* block_energies);

/* Packed VMC runs (no counterpart in the reference, which runs one input per
 * process): the VMC runs of n contexts (each alea_gpu_vmc_run's arguments:
 * cfgs[i] for ctxs[i]) stepped together on the first context's device, the
 * walkers of every run swept in one launch per step (one per sweep body:
 * the one-warp body for the systems that take it, a 32-thread generic body
 * for the rest), uneven walker counts and particle numbers packed raggedly.
 * Each run's blocks, energy, error, variance and acceptance equal its
 * alea_gpu_vmc_run's on its own context (same random streams, same walker
 * arithmetic; statuses[i] its status), so a run's result does not depend on
 * what it was packed with.  The launch shape (one CTA per walker or
 * persistent CTAs) comes from timing both on the first steps, per device;
 * once the set of running contexts repeats, a step is a CUDA graph replay.
 * Estimators and FP32 contexts are not packed (ALEA_ERR_UNSUPPORTED). */
int alea_gpu_vmc_run_packed(alea_gpu_ctx* const* ctxs, int n, const alea_gpu_run_config* cfgs,
                            alea_gpu_run_result* results, int* statuses);

/* Device time of the last alea_gpu_*_step / advance call's sweep kernel, in
 * milliseconds (CUDA events on the context's stream). */
int alea_gpu_last_kernel_ms(const alea_gpu_ctx* ctx, double* ms);

/* The cudaStream_t every call of this context is ordered on (no counterpart
 * in the reference: a host that times or overlaps work records its events
 * on this stream). */
int alea_gpu_stream(const alea_gpu_ctx* ctx, void** stream);
/* Bytes this context has copied host->device and device->host so far
 * (instrumentation; no counterpart in the reference). */
int alea_gpu_transfer_bytes(const alea_gpu_ctx* ctx, uint64_t* h2d, uint64_t* d2h);
/* Kernels this context has launched so far (instrumentation; no counterpart
 * in the reference). */
int alea_gpu_launch_count(const alea_gpu_ctx* ctx, uint64_t* launches);
/* Measured FP64 CUDA-core FMA throughput of a device in TFLOP/s (a
 * register-only loop of independent FMAs over every SM; instrumentation, no
 * counterpart in the reference): the roof of the FP64-latency-bound sweep. */
int alea_gpu_measure_fp64_peak(int device, double* tflops);

/* ───────────────────────── parameter derivatives ───────────────────────
 *
 * O_k = d ln psi / d p_k of every optimisable parameter — the shared widths
 * of Gaussian orbital blocks (opt_alpha), then the pair Jastrow terms' (their
 * n_opt / opt_index) — for every walker: what the linear method
 * samples (TrialWavefunction::compute_parameter_derivatives,
 * src/wavefunction/trial_wavefunction.h:104-114; PadeJastrow,
 * src/wavefunction/pade_jastrow.cpp:641-800 with its image sum,
 * periodic_pair_sum.cpp:80-92 and kspace_pair_sum.cpp:303-313;
 * DrummondJastrow, src/wavefunction/drummond_jastrow.cpp:201-320).
 * (SlaterDeterminant, src/wavefunction/slater_determinant.cpp:98-157 and,
 * for the curvature term below, :159-250).
 * derivs [n_params][nw]: blocks, then terms, parameter order within a term;
 * *n_params receives their number (derivs may be NULL to ask for it).  The
 * walkers must be evaluated (after upload, a step or alea_gpu_measure).
 * Backflow parameters are not computed here. */
int alea_gpu_parameter_derivatives(alea_gpu_ctx* ctx, double* derivs, int* n_params);
/* d(grad_d ln psi)/d p_k and d(lap_d ln psi)/d p_k of the same parameters,
 * [n_params][n_particles * dim][nw] each (the gradient planes' layout per
 * parameter): the curvature term of the linear method's Hbar
 * (compute_parameter_gradient_derivatives,
 * src/wavefunction/wavefunction_component.h:173-191; Padé
 * src/wavefunction/pade_jastrow.cpp:806-880 with the image sum's
 * kspace_pair_sum.cpp:315-320).  Either output may be NULL. */
int alea_gpu_parameter_gradient_derivatives(alea_gpu_ctx* ctx, double* dgrad, double* dlap, int* n_params);

/* ───────────────────────── configurations and carry-over ───────────────
 *
 * The walker population as the rows a checkpoint stores and the next driver
 * is seeded from: AoS [w][p][d] (io::WalkerFile, src/io/walker_io.h:34-40).
 * The reference hands configurations from one driver to the next through
 * the host (carry_over_walkers, src/qmc/app.cpp:1078-1098); here the rows can
 * stay in device memory, and a chain of stages on one system (VMC -> DMC tau1
 * -> DMC tau2) can keep the walkers' whole state. */

/* Final configurations, AoS rows [w][p][d] of n_particles x dim doubles per
 * walker (Driver::final_configurations, src/qmc/vmc.h:63-67 and
 * src/qmc/dmc.h:128-132; WalkerSet::append_configurations,
 * src/population/walker_set.cpp:253-262).  *nw receives the walker count;
 * rows may be NULL to ask for it. */
int alea_gpu_final_configurations(alea_gpu_ctx* ctx, double* rows, int* nw);
/* nw fresh walkers from n_rows AoS rows, walker w taking row w mod n_rows
 * (seed_walker_rows, src/qmc/app.cpp:1068-1076: a checkpoint's rows or the
 * previous driver's), wrapped and fully evaluated, weights 1: a driver's
 * reload_configurations (src/qmc/driver.h:55-58).  The checkpoint's
 * geometry and cell checks (app.cpp:834-866) are the host's. */
int alea_gpu_seed_walker_rows(alea_gpu_ctx* ctx, const double* rows, int n_rows, int nw);

/* Milestone checkpoints of alea_gpu_dmc_run (DMC::set_checkpoint_hook,
 * src/qmc/dmc.h:150-165; called at src/qmc/dmc.cpp:779 and :810-821): after
 * equilibration (tag "eq", blocks_done 0) and after 25/50/75% of the
 * accumulation blocks ("a25"/"a50"/"a75", integer quarters, each tag at most
 * once), between blocks.  The hook may call alea_gpu_final_configurations on
 * the context to write a snapshot (the reference's App writes
 * "<walkers_out>.<tag>.h5", app.cpp:885-911).  fn NULL: no hook. */
typedef void (*alea_gpu_checkpoint_fn)(void* user, alea_gpu_ctx* ctx, const char* tag, int blocks_done);
int alea_gpu_set_checkpoint_hook(alea_gpu_ctx* ctx, alea_gpu_checkpoint_fn fn, void* user);

enum { ALEA_CARRY_POSITIONS = 0, ALEA_CARRY_STATE = 1 };
/* Carry `from`'s population into `to` (nw walkers, walker w from source
 * walker w mod from's count) without a host round trip:
 *   ALEA_CARRY_POSITIONS  positions only, then a full evaluation in `to`
 *                         (the reference's semantics; any two systems with
 *                         the same particle count);
 *   ALEA_CARRY_STATE      the whole walker records (inverses, orbital rows,
 *                         ρ(k), ln ψ, derivatives, E_L), so the next stage
 *                         starts without re-evaluating; both contexts must be
 *                         created from identical systems (same tables, same
 *                         precision), else ALEA_ERR_INVALID.
 * Either way the walkers restart as a fresh ensemble: weight 1, age 0, no
 * ancestry.  The contexts may live on different devices (peer copy). */
int alea_gpu_carry_over(alea_gpu_ctx* from, alea_gpu_ctx* to, int nw, int mode);

/* ───────────────────────── estimators ──────────────────────────────────
 *
 * Observable estimators accumulated on the device from the walker records
 * (the reference's Estimator, src/estimators/estimator.h:44-131, whose
 * per-block lifecycle start_block → accumulate × n_steps → stop_block these
 * calls keep): pair correlation g(r) (PairCorrelation,
 * src/estimators/pair_correlation.cpp), the density grid (Density,
 * src/estimators/density.cpp) and the structure factor S(k) with the group
 * densities ρ_g(k) (StructureFactor, src/estimators/structure_factor.cpp).
 * A measurement bins every walker's configuration on the device, so a run
 * with estimators downloads nothing per step; a block's estimate (the array
 * the reference's stop_block stores) is read back once per block.
 *
 * Chains: a measurement may split the walkers into n_chains contiguous even
 * ranges, each with its own running block, as the reference's VMC keeps one
 * estimator clone per thread (src/qmc/vmc.cpp:201-207, reduced at :381-387).
 * Blocks are returned chain-major, the order in which the reference's
 * collect() concatenates the clones' histories.
 *
 * Block estimates (block_width doubles each, W = Σ weights of the block):
 *   gofr     [pair (a<=b)][bin]  histogram / W                (pair_correlation.cpp:143-160)
 *   density  [series][cell]      histogram / (W · V_cell)     (density.cpp:153-188)
 *   sofk     [pair][shell] S, then [group][k] Re ρ, then [group][k] Im ρ, each / W
 *                                                             (structure_factor.cpp:133-163)
 * Normalisation into g(r), errors and the named series are the host's
 * (the reference's finalize()). */
enum { ALEA_EST_GOFR = 1, ALEA_EST_DENSITY = 2, ALEA_EST_SOFK = 3 };

typedef struct {
    int kind;            /* ALEA_EST_* */
    int n_bins;          /* gofr: radial bins; density: bins per axis */
    double rmax;         /* gofr: range (at most the Wigner-Seitz inradius of a periodic cell);
                          * density: half-width of the box of an open cell */
    int per_particle;    /* density: one series per particle instead of per group */
    double kmax;         /* sofk: |k| <= kmax (periodic 2-D cells) */
} alea_gpu_estimator_spec;

typedef struct {
    int kind;
    int block_width;     /* doubles per block estimate */
    int n_chains;        /* chains of the current measurements (0 before the first) */
    int n_blocks;        /* finished blocks per chain */
    int n_series;        /* gofr, sofk: group pairs a <= b; density: groups or particles */
    int n_bins;
    int n_cells;         /* density: cells per series (n_bins^2) */
    int n_k, n_shells;   /* sofk */
    double volume;       /* cell area (0 for an open cell) */
    double cell_volume;  /* density: area of one grid cell */
} alea_gpu_estimator_desc;

/* Add an estimator (ALEA_ERR_INVALID for a gofr range beyond the
 * Wigner-Seitz inradius, S(k) on an open cell, or no k below kmax; the
 * reference's constructors throw there). */
int alea_gpu_add_estimator(alea_gpu_ctx* ctx, const alea_gpu_estimator_spec* spec, int* id);
/* Remove every estimator. */
int alea_gpu_clear_estimators(alea_gpu_ctx* ctx);
/* Drop every estimator's finished blocks and running block and its chain
 * count (a fresh clone of each). */
int alea_gpu_estimators_reset(alea_gpu_ctx* ctx);
/* Zero the running block of every estimator. */
int alea_gpu_estimators_start_block(alea_gpu_ctx* ctx);
/* One measurement of every estimator on the current walkers:
 * Estimator::accumulate(configs, weights).  weights [nw] (host, borrowed;
 * NULL: the walkers' own weights, 1 in VMC, the DMC weights between advance
 * and branch).  n_chains (>= 1) must stay the same until the next reset. */
int alea_gpu_estimators_accumulate(alea_gpu_ctx* ctx, const double* weights, int n_chains);
/* Close the running block of every estimator on every chain. */
int alea_gpu_estimators_stop_block(alea_gpu_ctx* ctx);
int alea_gpu_estimator_info(const alea_gpu_ctx* ctx, int id, alea_gpu_estimator_desc* out);
/* Finished block estimates, [n_chains][n_blocks][block_width]. */
int alea_gpu_estimator_blocks(const alea_gpu_ctx* ctx, int id, double* blocks);
/* The S(k) k set: k = n1 b1 + n2 b2 over the half space, sorted by |k|
 * (ties in (n1, n2) order), shells of equal |k|; any pointer may be NULL. */
int alea_gpu_estimator_kvectors(const alea_gpu_ctx* ctx, int id, int* n1, int* n2, double* kx, double* ky,
                                int* shell_of, double* shell_k, int* shell_count);

/* ───────────────────────── forward walking ─────────────────────────────
 *
 * Pure estimators of a DMC run (ForwardWalking, src/qmc/forward_walking.h:
 * Casulleras & Boronat, PRB 52, 3654 (1995)): every `interval` steps the
 * population's positions are stored (a snapshot, here in device memory); each
 * live walker's ancestor in every snapshot is carried through the branches;
 * at an accumulation step, for each lag T whose snapshot is T old, the
 * ancestors are weighted by the weight their descendants carry now and
 * measured: the potential energy (the pure potential; the pure kinetic energy
 * is E − ⟨V⟩) and the lag's pure estimators.  alea_gpu_dmc_run runs it when
 * set; the schedule follows DMC::DMC (src/qmc/dmc.cpp:102-138): lags are
 * whole numbers of steps of τ·n_substeps, the largest at most the
 * equilibration, interval divides n_steps — else the run fails with
 * ALEA_ERR_INVALID.  Steps count from the first equilibration step; a run
 * clears the previous results. */
typedef struct {
    double lag_time;              /* imaginary time T */
    int lag_steps;                /* T in DMC steps */
    int n_blocks;                 /* accumulation blocks with measurements */
    int64_t measurements;
    double surviving_fraction;    /* mean fraction of snapshot walkers with descendants */
    double potential, potential_error;   /* pure ⟨V⟩ and its reblocked error */
} alea_gpu_fw_summary;

/* lags [n_lags] strictly increasing imaginary times (n_lags = 0: off). */
int alea_gpu_set_forward_walking(alea_gpu_ctx* ctx, const double* lags, int n_lags, int interval);
/* A pure estimator measured at lag index `lag` (the estimator kinds above). */
int alea_gpu_add_fw_estimator(alea_gpu_ctx* ctx, int lag, const alea_gpu_estimator_spec* spec, int* id);
/* Results of lag index `lag` after a run; block_potentials (nullable) gets
 * one ⟨V⟩ per accumulation block (the reference's acc_block_potential_fw<i>). */
int alea_gpu_fw_result(const alea_gpu_ctx* ctx, int lag, alea_gpu_fw_summary* out, double* block_potentials);
int alea_gpu_fw_estimator_info(const alea_gpu_ctx* ctx, int lag, int id, alea_gpu_estimator_desc* out);
int alea_gpu_fw_estimator_blocks(const alea_gpu_ctx* ctx, int lag, int id, double* blocks);
int alea_gpu_fw_estimator_kvectors(const alea_gpu_ctx* ctx, int lag, int id, int* n1, int* n2, double* kx,
                                   double* ky, int* shell_of, double* shell_k, int* shell_count);

/* ── Host setup ─────────────────────────────────────────────────────────
 * Builds an alea_gpu_system (and its JSON description) for the systems the
 * reference's App assembles from a config, computing the same tables on the
 * host: cell from r_s (src/qmc/app.cpp:288-336), plane-wave shells
 * (src/wavefunction/orbital_set.h:575-665), Kato cusps
 * (src/builders/jastrow.cpp:48-98), the optimized Ewald breakup
 * (src/numerics/ewald_breakup.cpp:205-276, n_knots ladder of
 * src/hamiltonian/ewald_term.cpp) and the image-summed Padé
 * (src/wavefunction/periodic_pair_sum.cpp:21-60).  The setup owns every
 * table the system points to; free it after alea_gpu_create. */
typedef struct alea_gpu_setup alea_gpu_setup;

/* 2-D electron gas: n_up + n_down electrons at density rs in a square cell,
 * Padé u = a r/(1 + pade_b r) per spin pair (a from the cusp when pade_a <= 0),
 * Ewald tolerance ewald_tol (<= 0: 1e-6).  err receives a message on failure. */
int alea_gpu_setup_heg2d(int n_up, int n_down, double rs, double pade_b, double pade_a,
                         double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len);
/* The same electron gas at twist (twist_x, twist_y) in units of the
 * reciprocal vectors: twisted plane waves e^{i(k+θ)·r} filling the n lowest
 * |k + θ| per spin, a complex determinant (fixed-phase DMC); an integer twist
 * is Γ and gives the real determinant above.  ALEA_ERR_INVALID when a spin's
 * count splits a degenerate |k + θ| shell (builders/slater.cpp:244-262,
 * wavefunction/complex_orbital_set.h:278-343). */
int alea_gpu_setup_heg2d_twisted(int n_up, int n_down, double rs, double pade_b, double pade_a,
                                 double twist_x, double twist_y, double ewald_tol, alea_gpu_setup** out,
                                 char* err, size_t err_len);
/* 2-D Wigner crystal of nx × ny triangular sites (ny even), Gaussian
 * orbitals exp(-(gauss_c / rs²) |r - R|²), Drummond Jastrows with alpha0 and
 * cutoff cutoff_frac × the Wigner-Seitz radius (<= 0: 0.999), initial
 * jitter (<= 0: 1/sqrt(4 gauss_c / rs²)). */
int alea_gpu_setup_crystal2d(int nx, int ny, double rs, double gauss_c, double alpha0,
                             double cutoff_frac, double jitter, double ewald_tol,
                             alea_gpu_setup** out, char* err, size_t err_len);
/* Point charges in a periodic 2-D cell (rows of `lattice`, reduced as the
 * device reduces them) with Ewald Coulomb only: n_groups consecutive groups
 * of counts[g] particles of charge charges[g].  E_L is the electrostatic
 * energy (src/hamiltonian/ewald_term.cpp:368-612). */
int alea_gpu_setup_charges2d(const double* lattice, int n_groups, const int* counts, const double* charges,
                             double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len);
/* The 3-D Coulomb Ewald tables of a periodic cell (no counterpart in the
 * reference, which refuses 3-D Ewald: src/numerics/ewald_breakup.cpp:211-213):
 * rows a_i of `lattice` (9 numbers), the optimized breakup of 1/r with the
 * 3-D radial kernel, r_c the Wigner-Seitz inradius.  Host tables only, in
 * alea_gpu_setup_json (the spline, half-space k-vectors with weights f̃_l/V,
 * f_l(0), f̃_s(0)/V).  The system of a 3-D electron gas that uses these
 * tables is alea_gpu_setup_heg3d's. */
int alea_gpu_setup_ewald3d(const double* lattice, double ewald_tol, alea_gpu_setup** out, char* err,
                           size_t err_len);
/* 3-D electron gas with backflow (no counterpart among the reference's
 * builders, which refuse 3-D plane-wave shells and 3-D Ewald; its backflow
 * determinant, BackflowSlaterDeterminant, src/wavefunction/
 * backflow_slater_determinant.h:15-80, is dimension-generic): n_up + n_down
 * electrons in a cubic cell of volume N 4π rs³/3, one backflow determinant of
 * real plane waves per spin (k = 2π n/L by |n|², then lexicographic n, k = 0
 * first, cos then sin per ±n), channels from the own spin (c_0 = bf_like,
 * c_1 = 3 c_0/L) and the other spin (c_0 = bf_unlike), C = 3, L = bf_cut
 * (<= 0: half the side); Drummond Jastrows (C = 3, the 3-D Kato cusps 1/2 and
 * 1/4, alpha0, cutoff 0.999 × half the side); the 3-D Ewald sum of
 * alea_gpu_setup_ewald3d. */
int alea_gpu_setup_heg3d(int n_up, int n_down, double rs, double bf_like, double bf_unlike, double bf_cut,
                         double alpha0, double ewald_tol, alea_gpu_setup** out, char* err, size_t err_len);
/* 2-D dipolar bosons: n of mass 1 in a hexagonal cell at density rs, C/r^p
 * (strength, exponent) with its continuum tail, and the zero-energy Jastrow
 * with the given matching radius, cut off at the Wigner-Seitz inradius. */
int alea_gpu_setup_dipoles2d(int n, double rs, double strength, double exponent, double matching_radius,
                             alea_gpu_setup** out, char* err, size_t err_len);
/* Open 2-D exciton with the exact trial function (E = -1). */
int alea_gpu_setup_exciton2d(double L_init, alea_gpu_setup** out);
const alea_gpu_system* alea_gpu_setup_system(const alea_gpu_setup* s);
const char* alea_gpu_setup_json(const alea_gpu_setup* s);
/* Initial walkers, AoS [w][p][d], with App::initialize_positions' draws
 * (src/qmc/app.cpp:56-112): one mt19937_64 seeded with `seed`. */
int alea_gpu_setup_positions(const alea_gpu_setup* s, uint64_t seed, int nw, double* positions);
void alea_gpu_setup_free(alea_gpu_setup* s);

/* ───────────────────────── precision ───────────────────────────────────
 *
 * No reference counterpart (the reference is FP64 throughout).  FP64 is the
 * drop-in.  ALEA_PRECISION_FP32 makes the sweep entry points (vmc_step,
 * dmc_advance, the runs, the allocation-free step) run the FP32 form: the
 * inverses, orbitals, ratios, rank-one updates, pair-Jastrow radial terms and
 * image-sum terms of every move in FP32 (angles reduced in FP64, sums in
 * FP64); positions, the Jastrow gradient planes, ρ(k), the inverse
 * recomputation every 64 updates (rows recomputed in FP64, Gauss-Jordan in
 * FP64), log|det|, the local energy and the DMC weights in FP64.  For
 * real plane-wave determinants with Padé or Drummond pair terms, ≤ 64
 * particles (the electron gases); ALEA_ERR_UNSUPPORTED otherwise.  The FP32 form keeps no FP64
 * orbital rows, so meanwhile alea_gpu_measure re-evaluates the walkers and
 * alea_gpu_move is refused; setting FP64 again re-evaluates them. */
enum { ALEA_PRECISION_FP64 = 0, ALEA_PRECISION_FP32 = 1 };
int alea_gpu_set_precision(alea_gpu_ctx* ctx, int precision);

/* ───────────────────────── serving ─────────────────────────────────────
 *
 * No reference counterpart: the reference runs one input file per process.
 * A server takes VMC / DMC jobs that differ in system, walkers and length,
 * keeps each admitted job's walkers and inverses on the device in a context
 * of its own (own CUDA stream, own random streams keyed by the job's seed),
 * and runs up to max_running of them at once, so their kernels overlap on
 * the device.  A job is admitted, in arrival order among those that fit,
 * when its device footprint (≈ 2 × capacity × record bytes, the record being
 * Σ_blocks 6 N_b² + 14 N + … doubles) fits the HBM budget left by the running
 * ones; jobs that arrive while others run are admitted as slots and memory
 * free up.  A job's result does not depend on what else runs: its arithmetic
 * is that of alea_gpu_vmc_run / alea_gpu_dmc_run on its own context.
 *
 * Threads: any host thread may submit, poll or cancel; the server's worker
 * threads own the contexts.  Borrowed pointers (system tables, positions)
 * must stay valid until the job is done, failed or cancelled. */
typedef struct alea_gpu_server alea_gpu_server;

enum { ALEA_JOB_VMC = 0, ALEA_JOB_DMC = 1 };

typedef struct {
    const alea_gpu_system* system;   /* borrowed */
    const double* positions;         /* AoS [w][p][d] initial walkers, borrowed */
    int n_walkers;
    int mode;                        /* ALEA_JOB_VMC or ALEA_JOB_DMC */
    alea_gpu_run_config run;         /* as for alea_gpu_vmc_run / alea_gpu_dmc_run */
} alea_gpu_job;

typedef struct {
    int status;                      /* ALEA_OK or the job's ALEA_ERR_* code */
    alea_gpu_run_result result;
    double queue_ms;                 /* submission to admission */
    double run_ms;                   /* admission to completion */
    double latency_ms;               /* submission to completion */
    size_t footprint_bytes;          /* the admission estimate */
} alea_gpu_job_result;

/* hbm_budget_bytes = 0: 80% of the device memory free at creation;
 * max_running >= 1 worker contexts. */
int alea_gpu_server_create(int device, size_t hbm_budget_bytes, int max_running, alea_gpu_server** out);
/* The same server with its VMC jobs packed (no counterpart in the reference):
 * two preparer threads admit queued VMC jobs as the budget frees up and
 * build their contexts; one packing thread per sweep body (one-warp real or
 * complex, generic of 32, 64 or 128 threads) steps its admitted jobs
 * together, all their walkers in one sweep launch per step
 * (alea_gpu_vmc_run_packed), independently of the other bodies; a job's
 * result equals its alea_gpu_vmc_run on its own context whatever else runs.
 * DMC jobs, and the VMC jobs of three-dimensional systems (the packed sweeps
 * are two-dimensional), take the max_running worker contexts as in
 * alea_gpu_server_create. */
int alea_gpu_server_create_packed(int device, size_t hbm_budget_bytes, int max_running, alea_gpu_server** out);
/* Queue a job; never blocks on the device.  ALEA_ERR_NOMEM when the job
 * alone exceeds the budget. */
int alea_gpu_submit_job(alea_gpu_server* s, const alea_gpu_job* job, uint64_t* job_id);
/* Wait at most timeout_ms (0: do not wait) for a job: ALEA_OK with *out
 * filled when it has finished (out->status tells how), ALEA_ERR_TIMEOUT when
 * it is still queued or running, ALEA_ERR_INVALID for an unknown id.  A
 * finished job's result is handed out once: the poll that returns it drops
 * the job, and later polls of its id return ALEA_ERR_INVALID. */
int alea_gpu_poll(alea_gpu_server* s, uint64_t job_id, int timeout_ms, alea_gpu_job_result* out);
/* Cancel a queued job at once, or a running one at its next step
 * (status ALEA_ERR_CANCELLED); ALEA_ERR_INVALID for an unknown or finished id. */
int alea_gpu_cancel(alea_gpu_server* s, uint64_t job_id);
/* Cancel what is left, join the workers, free every context. */
int alea_gpu_server_destroy(alea_gpu_server* s);
const char* alea_gpu_server_last_error(const alea_gpu_server* s);

#ifdef __cplusplus
}
#endif
#endif /* ALEA_GPU_H */
