"""ctypes binding of the C ABI in include/alea_gpu.h (libalea_b200.so).

The structures below mirror the header field for field.  The library is
built in-tree (``python -m alea_b200.build``); importing this module on a
machine without it raises ImportError rather than falling back to anything.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libalea_b200.so")

ALEA_OK = 0
ERRORS = {1: "invalid", 2: "cuda", 3: "unsupported", 4: "singular", 5: "timeout", 6: "nomem"}
ORB_PLANE_WAVE, ORB_GAUSSIAN, ORB_TWISTED_PLANE_WAVE = 0, 1, 2
PAIR_PADE, PAIR_DRUMMOND, PAIR_ZERO_ENERGY = 0, 1, 2
STREAM_VMC = 0x766D632D74687264
STREAM_DMC = 0x646D632D74687264
STREAM_BRANCH = 0x646D632D62726368

c_dp = ctypes.POINTER(ctypes.c_double)
c_ip = ctypes.POINTER(ctypes.c_int)
MAX_OPT = 4   # ALEA_GPU_MAX_OPT


class Spline(ctypes.Structure):
    _fields_ = [("r_cut", ctypes.c_double), ("inv_delta", ctypes.c_double),
                ("n_knots", ctypes.c_int), ("scaled", c_dp)]


class KSet(ctypes.Structure):
    _fields_ = [("n_k", ctypes.c_int), ("n1", c_ip), ("n2", c_ip), ("kx", c_dp),
                ("ky", c_dp), ("weight", c_dp), ("n3", c_ip), ("kz", c_dp)]


class Group(ctypes.Structure):
    _fields_ = [("first", ctypes.c_int), ("last", ctypes.c_int), ("charge", ctypes.c_double),
                ("inv_mass", ctypes.c_double * 3)]


class Orbitals(ctypes.Structure):
    _fields_ = [("first", ctypes.c_int), ("last", ctypes.c_int), ("type", ctypes.c_int),
                ("k", c_dp), ("is_sin", c_ip), ("centers", c_dp), ("alphas", c_dp),
                ("opt_alpha", ctypes.c_int)]


class PairTerm(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n_pairs", ctypes.c_int),
                ("pairs", (ctypes.c_int * 4) * 4), ("num_order", ctypes.c_int),
                ("den_order", ctypes.c_int), ("coeffs", ctypes.c_double * 16),
                ("image_sum", ctypes.c_int), ("short_range", Spline), ("u_inf", ctypes.c_double),
                ("kset", KSet), ("C", ctypes.c_int), ("gamma", ctypes.c_double),
                ("L", ctypes.c_double), ("n_coeffs", ctypes.c_int),
                ("dcoeffs", ctypes.c_double * 16), ("ze_b", ctypes.c_double),
                ("ze_exponent", ctypes.c_double), ("ze_matching_radius", ctypes.c_double),
                ("ze_cutoff", ctypes.c_double), ("n_opt", ctypes.c_int), ("opt_index", ctypes.c_int * MAX_OPT),
                ("opt_inf", ctypes.c_double * 4), ("opt_short_range", Spline * 4),
                ("opt_weight", c_dp * 4)]


class Ewald(ctypes.Structure):
    _fields_ = [("enabled", ctypes.c_int), ("r_cut", ctypes.c_double),
                ("inv_eps", ctypes.c_double), ("constant", ctypes.c_double),
                ("long_range", Spline), ("kset", KSet)]


class Coulomb(ctypes.Structure):
    _fields_ = [("a_first", ctypes.c_int), ("a_last", ctypes.c_int), ("b_first", ctypes.c_int),
                ("b_last", ctypes.c_int), ("coef", ctypes.c_double)]


class InversePower(ctypes.Structure):
    _fields_ = [("a_first", ctypes.c_int), ("a_last", ctypes.c_int), ("b_first", ctypes.c_int),
                ("b_last", ctypes.c_int), ("strength", ctypes.c_double),
                ("exponent", ctypes.c_double), ("tail", ctypes.c_double)]


class BackflowChannel(ctypes.Structure):
    _fields_ = [("source_first", ctypes.c_int), ("source_last", ctypes.c_int), ("C", ctypes.c_int),
                ("L", ctypes.c_double), ("n_coeffs", ctypes.c_int), ("coeffs", ctypes.c_double * 16),
                ("zero_slope", ctypes.c_int), ("n_opt", ctypes.c_int), ("opt_index", ctypes.c_int * MAX_OPT)]


class Backflow(ctypes.Structure):
    _fields_ = [("first", ctypes.c_int), ("last", ctypes.c_int), ("type", ctypes.c_int),
                ("k", c_dp), ("is_sin", c_ip), ("centers", c_dp), ("alphas", c_dp),
                ("n_channels", ctypes.c_int), ("channels", BackflowChannel * 4)]


class System(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n_particles", ctypes.c_int), ("periodic", ctypes.c_int),
                ("lattice", ctypes.c_double * 9), ("n_groups", ctypes.c_int),
                ("groups", Group * 8), ("n_blocks", ctypes.c_int), ("blocks", Orbitals * 4),
                ("n_terms", ctypes.c_int), ("terms", PairTerm * 8), ("ewald", Ewald),
                ("n_coulomb", ctypes.c_int), ("coulomb", Coulomb * 8), ("n_inverse_power", ctypes.c_int),
                ("inverse_power", InversePower * 8), ("n_backflow", ctypes.c_int),
                ("backflow", Backflow * 2)]


class VmcParams(ctypes.Structure):
    _fields_ = [("tau", ctypes.c_double), ("n_substeps", ctypes.c_int), ("use_drift", ctypes.c_int)]


class StepStats(ctypes.Structure):
    _fields_ = [("energy_sum", ctypes.c_double), ("energy_sq_sum", ctypes.c_double),
                ("weight_sum", ctypes.c_double), ("n_accepted", ctypes.c_int64),
                ("n_proposed", ctypes.c_int64), ("n_cut", ctypes.c_int64),
                ("n_walkers", ctypes.c_int)]


class DmcParams(ctypes.Structure):
    _fields_ = [("tau", ctypes.c_double), ("n_substeps", ctypes.c_int),
                ("e_trial", ctypes.c_double), ("e_ref", ctypes.c_double),
                ("e_cut", ctypes.c_double), ("e_max", ctypes.c_double)]


class RunConfig(ctypes.Structure):
    _fields_ = [("n_equilibration_blocks", ctypes.c_int), ("n_accumulation_blocks", ctypes.c_int),
                ("n_steps", ctypes.c_int), ("n_substeps", ctypes.c_int), ("tau", ctypes.c_double),
                ("use_drift", ctypes.c_int), ("n_streams", ctypes.c_int), ("seed", ctypes.c_uint64),
                ("target_walkers", ctypes.c_int), ("population_generations", ctypes.c_double),
                ("branch_cutoff_alpha", ctypes.c_double)]


class RunResult(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("energy_error", ctypes.c_double),
                ("variance", ctypes.c_double), ("acceptance", ctypes.c_double),
                ("walltime_s", ctypes.c_double), ("n_walkers", ctypes.c_int),
                ("e_trial", ctypes.c_double), ("n_moves", ctypes.c_int64),
                ("n_evaluations", ctypes.c_int64)]


class Job(ctypes.Structure):
    _fields_ = [("system", ctypes.POINTER(System)), ("positions", c_dp), ("n_walkers", ctypes.c_int),
                ("mode", ctypes.c_int), ("run", RunConfig)]


class JobResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("result", RunResult), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("footprint_bytes", ctypes.c_size_t)]


class EstimatorSpec(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("n_bins", ctypes.c_int), ("rmax", ctypes.c_double),
                ("per_particle", ctypes.c_int), ("kmax", ctypes.c_double)]


class EstimatorDesc(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("block_width", ctypes.c_int), ("n_chains", ctypes.c_int),
                ("n_blocks", ctypes.c_int), ("n_series", ctypes.c_int), ("n_bins", ctypes.c_int),
                ("n_cells", ctypes.c_int), ("n_k", ctypes.c_int), ("n_shells", ctypes.c_int),
                ("volume", ctypes.c_double), ("cell_volume", ctypes.c_double)]


class FwSummary(ctypes.Structure):
    _fields_ = [("lag_time", ctypes.c_double), ("lag_steps", ctypes.c_int), ("n_blocks", ctypes.c_int),
                ("measurements", ctypes.c_int64), ("surviving_fraction", ctypes.c_double),
                ("potential", ctypes.c_double), ("potential_error", ctypes.c_double)]


EST_GOFR, EST_DENSITY, EST_SOFK = 1, 2, 3
CHECKPOINT_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int)
CARRY_POSITIONS, CARRY_STATE = 0, 1
JOB_VMC, JOB_DMC = 0, 1
PRECISION_FP64, PRECISION_FP32 = 0, 1
ERR_TIMEOUT, ERR_NOMEM, ERR_CANCELLED = 5, 6, 7


EXPORTS = [
    "alea_gpu_abi_version", "alea_gpu_create", "alea_gpu_destroy", "alea_gpu_last_error",
    "alea_gpu_upload_walkers", "alea_gpu_evaluate", "alea_gpu_num_walkers",
    "alea_gpu_download_walkers", "alea_gpu_move", "alea_gpu_measure", "alea_gpu_set_streams",
    "alea_gpu_vmc_step", "alea_gpu_dmc_advance", "alea_gpu_dmc_branch", "alea_gpu_vmc_run",
    "alea_gpu_dmc_run", "alea_gpu_last_kernel_ms", "alea_gpu_stream", "alea_gpu_transfer_bytes",
    "alea_gpu_launch_count", "alea_gpu_vmc_step_noalloc", "alea_gpu_download_phase",
    "alea_gpu_setup_heg2d", "alea_gpu_setup_heg2d_twisted", "alea_gpu_setup_crystal2d",
    "alea_gpu_setup_exciton2d",
    "alea_gpu_setup_charges2d", "alea_gpu_setup_dipoles2d", "alea_gpu_setup_ewald3d", "alea_gpu_setup_heg3d",
    "alea_gpu_setup_system", "alea_gpu_setup_json", "alea_gpu_setup_positions",
    "alea_gpu_setup_free",
    "alea_gpu_set_precision",
    "alea_gpu_server_create", "alea_gpu_submit_job", "alea_gpu_poll", "alea_gpu_cancel",
    "alea_gpu_server_destroy", "alea_gpu_server_last_error",
    "alea_gpu_add_estimator", "alea_gpu_clear_estimators", "alea_gpu_estimators_reset",
    "alea_gpu_estimators_start_block", "alea_gpu_estimators_accumulate", "alea_gpu_estimators_stop_block",
    "alea_gpu_estimator_info", "alea_gpu_estimator_blocks", "alea_gpu_estimator_kvectors",
    "alea_gpu_final_configurations", "alea_gpu_seed_walker_rows", "alea_gpu_carry_over",
    "alea_gpu_parameter_derivatives", "alea_gpu_parameter_gradient_derivatives", "alea_gpu_measure_fp64_peak",
    "alea_gpu_propose", "alea_gpu_ratio", "alea_gpu_commit", "alea_gpu_local_energy", "alea_gpu_set_rng_streams",
    "alea_gpu_vmc_steps", "alea_gpu_dmc_steps", "alea_gpu_set_checkpoint_hook",
    "alea_gpu_set_forward_walking", "alea_gpu_add_fw_estimator", "alea_gpu_fw_result",
    "alea_gpu_fw_estimator_info", "alea_gpu_fw_estimator_blocks", "alea_gpu_fw_estimator_kvectors",
    "alea_gpu_vmc_run_packed", "alea_gpu_server_create_packed",
]

_LIB = None


def load() -> ctypes.CDLL:
    """Load libalea_b200.so and declare the ABI's signatures."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m alea_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    P = ctypes.c_void_p
    I, D = ctypes.c_int, ctypes.c_double
    sig = {
        "alea_gpu_abi_version": ([], I),
        "alea_gpu_create": ([ctypes.POINTER(System), I, I, ctypes.POINTER(P)], I),
        "alea_gpu_destroy": ([P], I),
        "alea_gpu_last_error": ([P], ctypes.c_char_p),
        "alea_gpu_upload_walkers": ([P, c_dp, I], I),
        "alea_gpu_evaluate": ([P], I),
        "alea_gpu_num_walkers": ([P, c_ip], I),
        "alea_gpu_download_walkers": ([P, c_dp, c_dp, c_dp, c_dp, c_dp, c_dp], I),
        "alea_gpu_download_phase": ([P, c_dp, c_dp, c_dp], I),
        "alea_gpu_move": ([P, I, c_dp, ctypes.POINTER(ctypes.c_uint8), c_dp, c_dp, c_dp, c_dp], I),
        "alea_gpu_measure": ([P], I),
        "alea_gpu_set_streams": ([P, ctypes.c_uint64, ctypes.c_uint64, I], I),
        "alea_gpu_vmc_step": ([P, ctypes.POINTER(VmcParams), ctypes.POINTER(StepStats)], I),
        "alea_gpu_vmc_step_noalloc": ([P, ctypes.POINTER(VmcParams), ctypes.POINTER(StepStats)], I),
        "alea_gpu_dmc_advance": ([P, ctypes.POINTER(DmcParams), ctypes.POINTER(StepStats)], I),
        "alea_gpu_dmc_branch": ([P, ctypes.POINTER(ctypes.c_uint64), I], I),
        "alea_gpu_vmc_run": ([P, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult), c_dp], I),
        "alea_gpu_vmc_run_packed": ([ctypes.POINTER(P), I, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult),
                                     ctypes.POINTER(I)], I),
        "alea_gpu_dmc_run": ([P, ctypes.POINTER(RunConfig), ctypes.POINTER(RunResult), c_dp], I),
        "alea_gpu_last_kernel_ms": ([P, c_dp], I),
        "alea_gpu_stream": ([P, ctypes.POINTER(P)], I),
        "alea_gpu_launch_count": ([P, ctypes.POINTER(ctypes.c_uint64)], I),
        "alea_gpu_transfer_bytes": ([P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)], I),
        "alea_gpu_setup_heg2d": ([I, I, D, D, D, D, ctypes.POINTER(P), ctypes.c_char_p,
                                  ctypes.c_size_t], I),
        "alea_gpu_setup_heg2d_twisted": ([I, I, D, D, D, D, D, D, ctypes.POINTER(P), ctypes.c_char_p,
                                          ctypes.c_size_t], I),
        "alea_gpu_setup_crystal2d": ([I, I, D, D, D, D, D, D, ctypes.POINTER(P), ctypes.c_char_p,
                                      ctypes.c_size_t], I),
        "alea_gpu_setup_exciton2d": ([D, ctypes.POINTER(P)], I),
        "alea_gpu_setup_dipoles2d": ([I, D, D, D, D, ctypes.POINTER(P), ctypes.c_char_p, ctypes.c_size_t], I),
        "alea_gpu_setup_charges2d": ([c_dp, I, c_ip, c_dp, D, ctypes.POINTER(P), ctypes.c_char_p,
                                      ctypes.c_size_t], I),
        "alea_gpu_setup_ewald3d": ([c_dp, D, ctypes.POINTER(P), ctypes.c_char_p, ctypes.c_size_t], I),
        "alea_gpu_setup_heg3d": ([I, I, D, D, D, D, D, D, ctypes.POINTER(P), ctypes.c_char_p, ctypes.c_size_t], I),
        "alea_gpu_setup_system": ([P], ctypes.POINTER(System)),
        "alea_gpu_setup_json": ([P], ctypes.c_char_p),
        "alea_gpu_setup_positions": ([P, ctypes.c_uint64, I, c_dp], I),
        "alea_gpu_setup_free": ([P], None),
        "alea_gpu_set_precision": ([P, I], I),
        "alea_gpu_server_create": ([I, ctypes.c_size_t, I, ctypes.POINTER(P)], I),
        "alea_gpu_server_create_packed": ([I, ctypes.c_size_t, I, ctypes.POINTER(P)], I),
        "alea_gpu_submit_job": ([P, ctypes.POINTER(Job), ctypes.POINTER(ctypes.c_uint64)], I),
        "alea_gpu_poll": ([P, ctypes.c_uint64, I, ctypes.POINTER(JobResult)], I),
        "alea_gpu_cancel": ([P, ctypes.c_uint64], I),
        "alea_gpu_server_destroy": ([P], I),
        "alea_gpu_server_last_error": ([P], ctypes.c_char_p),
        "alea_gpu_parameter_derivatives": ([P, c_dp, c_ip], I),
        "alea_gpu_measure_fp64_peak": ([I, c_dp], I),
        "alea_gpu_set_checkpoint_hook": ([P, CHECKPOINT_FN, P], I),
        "alea_gpu_propose": ([P, I, c_dp], I),
        "alea_gpu_ratio": ([P, I, c_dp, c_dp, c_dp, c_dp], I),
        "alea_gpu_commit": ([P, I, ctypes.POINTER(ctypes.c_uint8)], I),
        "alea_gpu_local_energy": ([P, c_dp], I),
        "alea_gpu_set_rng_streams": ([P, ctypes.c_uint64, ctypes.c_uint64, I], I),
        "alea_gpu_vmc_steps": ([P, ctypes.POINTER(VmcParams), I, ctypes.POINTER(StepStats)], I),
        "alea_gpu_dmc_steps": ([P, ctypes.POINTER(DmcParams), I, ctypes.POINTER(ctypes.c_uint64), I,
                                ctypes.POINTER(StepStats)], I),
        "alea_gpu_parameter_gradient_derivatives": ([P, c_dp, c_dp, c_ip], I),
        "alea_gpu_set_forward_walking": ([P, c_dp, I, I], I),
        "alea_gpu_add_fw_estimator": ([P, I, ctypes.POINTER(EstimatorSpec), c_ip], I),
        "alea_gpu_fw_result": ([P, I, ctypes.POINTER(FwSummary), c_dp], I),
        "alea_gpu_fw_estimator_info": ([P, I, I, ctypes.POINTER(EstimatorDesc)], I),
        "alea_gpu_fw_estimator_blocks": ([P, I, I, c_dp], I),
        "alea_gpu_fw_estimator_kvectors": ([P, I, I, c_ip, c_ip, c_dp, c_dp, c_ip, c_dp, c_ip], I),
        "alea_gpu_final_configurations": ([P, c_dp, c_ip], I),
        "alea_gpu_seed_walker_rows": ([P, c_dp, I, I], I),
        "alea_gpu_carry_over": ([P, P, I, I], I),
        "alea_gpu_add_estimator": ([P, ctypes.POINTER(EstimatorSpec), c_ip], I),
        "alea_gpu_clear_estimators": ([P], I),
        "alea_gpu_estimators_reset": ([P], I),
        "alea_gpu_estimators_start_block": ([P], I),
        "alea_gpu_estimators_accumulate": ([P, c_dp, I], I),
        "alea_gpu_estimators_stop_block": ([P], I),
        "alea_gpu_estimator_info": ([P, I, ctypes.POINTER(EstimatorDesc)], I),
        "alea_gpu_estimator_blocks": ([P, I, c_dp], I),
        "alea_gpu_estimator_kvectors": ([P, I, c_ip, c_ip, c_dp, c_dp, c_ip, c_dp, c_ip], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib
