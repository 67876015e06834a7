#!/usr/bin/env python
"""Benchmark: fixed-node DMC of the 2-D electron gas on the B200 walker path.

Workload: N = 42 electrons (21 up / 21 down) at r_s = 30 in a square periodic
cell, plane-wave Slater determinants times an image-summed Padé Jastrow
(a from the Kato cusp, b = 0.3), 2-D Ewald Coulomb; 16384 walkers, τ = 0.5,
one sweep per step, population control toward 16384.  All arithmetic FP64.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one DMC generation: every walker sweeps its 42 electrons with
drift-diffusion moves, refreshes its derivatives, evaluates E_L and its branch
weight (one sweep kernel), then the population branches (host serial stream,
device gather).  `value` is electron-moves/s of K such steps with the walkers
resident in HBM, CUDA events on the context's stream; `e2e` is the same
metric through the C ABI's run call from pinned host positions, with the
upload, the run's per-step weight reads and branch maps, and the download of
positions and local energies inside the timed region.

Under torchrun each rank runs an independent replica (its own seed) on its
GPU; value = moves of all ranks / the slowest rank's time.

--impl reference times the reference's own OpenMP DMC (oracle/_ref, compiled
from the reference sources) on the host cores on a bounded walker sample.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_UP, N_DOWN, RS, PADE_B = 21, 21, 30.0, 0.3
NP = N_UP + N_DOWN
DIM = 2
TAU = 0.5
VMC_TAU = (0.5 * RS) ** 2          # Metropolis step 0.5 r_s for the pre-equilibration
GENERATIONS = 10.0
CUTOFF_ALPHA = 2.0
WORKLOAD = (f"DMC 2-D electron gas N={NP} ({N_UP} up/{N_DOWN} down) rs={RS:g}, "
            f"tau={TAU}, 1 sweep per step, FP64")
METRIC = "electron-moves/s"
UNIT = "moves/s"


def parse():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--walkers", type=int, default=16384)
    ap.add_argument("--pre", type=int, default=20, help="untimed VMC pre-equilibration steps")
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--cpu-walkers", type=int, default=4096,
                    help="walker sample of the host-CPU baseline")
    ap.add_argument("--cpu-steps", type=int, default=40,
                    help="timed DMC steps of the host-CPU baseline (about 10 s of the reference's work)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32-form measurement")
    ap.add_argument("--no-estimators", action="store_true",
                    help="skip the device-estimator (g(r), density, S(k)) measurement")
    ap.add_argument("--density-per-particle", action="store_true",
                    help="measure the density per particle (one 48x48 grid each) instead of per spin")
    ap.add_argument("--serve", action="store_true",
                    help="serving mix instead of the DMC step: Poisson VMC jobs through alea_gpu_server")
    ap.add_argument("--serve-jobs", type=int, default=60)
    ap.add_argument("--serve-rate", type=float, default=50.0, help="arrivals per second")
    ap.add_argument("--serve-slots", type=int, default=8, help="DMC jobs running at once (worker contexts)")
    ap.add_argument("--serve-unpacked", action="store_true",
                    help="one context and launch stream per job instead of the packed scheduler")
    ap.add_argument("--no-other-systems", dest="other_systems", action="store_false",
                    help="skip the twisted and backflow variants of the gas")
    ap.add_argument("--vmc-blocks", type=int, default=100,
                    help="blocks of 50 sweeps of the VMC sub-object (512 walkers; 0: none)")
    ap.add_argument("--serve-bench-jobs", type=int, default=24,
                    help="jobs of the serving sub-object of the default line (0: none)")
    return ap.parse_args()


# ───────────────────────── algorithmic work per unit ─────────────────────

def work_per_unit(desc):
    """Bytes per electron-move (state streamed once per sweep, per move) and
    per local-energy evaluation, from the system's sizes."""
    blocks = [b["last"] - b["first"] for b in desc["slater"]]
    n_g = len(desc["groups"])
    n_kj = max((len(p["image_sum"]["weight"]) for p in desc.get("pade", []) if "image_sum" in p),
               default=0)
    s_w = (sum(n * n for n in blocks) + NP * DIM + NP * (NP - 1) // 2 + 2 * NP * DIM
           + 2 * n_g * n_kj + 4)
    b_move = 2.0 * 8.0 * s_w / NP
    b_eval = 8.0 * (NP * (NP - 1) / 2 + 3 * NP * DIM + 2)
    return b_move, b_eval, n_kj, len(desc["ewald"]["weight"])


# ───────────────────────── measured peaks, clocks ───────────────────────

def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of one GPU's clocks during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_id: str | None):
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if device_id:
            cmd += ["-i", device_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 8:
                continue
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except ValueError:
                continue
            for name, v in zip(names, r[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def profiled_traffic_per_walker():
    """DRAM bytes per walker per sweep-kernel launch from the committed ncu
    summary of that kernel (a `dram_bytes_per_walker:` line), or None."""
    path = os.path.join(ROOT, "profiles", "sweep_dmc_heg42.md")
    try:
        for line in open(path):
            if line.strip().startswith("dram_bytes_per_walker:"):
                return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


# ───────────────────────── reference (host CPU) arm ─────────────────────

def profiled_fp64_flops_per_move():
    """FP64 flops per move of the sweep kernel from the committed ncu summary
    (a `fp64_flops_per_move:` line), or None."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "sweep_dmc_heg42.md")
    try:
        for line in open(path):
            if line.strip().startswith("fp64_flops_per_move:"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_cpu(nw: int, steps: int, warmup: int, seed: int):
    """Reference OpenMP DMC on the host cores: returns (moves/s, info)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    threads = host_threads()
    if os.path.exists(harness):
        args = [harness, "bench", "system=heg", f"nu={N_UP}", f"nd={N_DOWN}", f"rs={RS:g}",
                f"b={PADE_B:g}", f"nw={nw}", f"steps={warmup + steps + 1}", f"tau={TAU}",
                f"seed={seed}", f"threads={threads}"]
        out = subprocess.run(args, capture_output=True, text=True, check=True,
                             env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
        d = json.loads(out.stdout)
        stamps = np.array(d["stamps"])
        walkers = np.array(d["walkers"])
        dt = np.diff(stamps)[warmup:warmup + steps]
        moves = float(np.sum(walkers[warmup + 1:warmup + 1 + steps])) * NP
        return moves / float(np.sum(dt)), {"kind": "reference", "cores": int(d["threads"]),
                                           "sample": f"{nw} walkers x {steps} DMC steps "
                                                     f"(after {warmup} untimed), same system"}
    # the compiled reference is absent: the oracle restatement (one thread)
    from oracle import Oracle
    from alea_b200 import setup as S
    st = S.heg2d(N_UP, N_DOWN, RS, PADE_B)
    o = Oracle(st.desc)
    o.init(st.positions(seed, nw), capacity=2 * nw + 2)
    t0 = time.perf_counter()
    o.dmc(1, seed, 0, 1, steps, 1, TAU, nw)
    dt = time.perf_counter() - t0
    return nw * NP * steps / dt, {"kind": "port", "cores": 1,
                                  "sample": f"{nw} walkers x {steps} DMC steps, oracle restatement"}


def reference_vmc_3d(nw: int, steps: int, seed: int):
    """The compiled reference's VMC of the 3-D backflow gas on the host cores
    (its own BackflowSlaterDeterminant, Drummond Jastrow and drivers; kinetic
    energy only, since it has no 3-D Ewald sum): moves/s over `steps` sweeps
    after one untimed sweep, or None without the compiled reference."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        return None
    threads = host_threads()
    args = [harness, "bench", "method=vmc", "system=heg3d", "nu=27", "nd=27", "rs=5", "alpha0=-0.01",
            f"nw={nw}", f"steps={steps + 1}", "tau=1.0", f"seed={seed}", f"threads={threads}"]
    out = subprocess.run(args, capture_output=True, text=True, check=True,
                         env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
    d = json.loads(out.stdout)
    dt = float(np.sum(np.diff(np.array(d["stamps"]))[-steps:]))
    return {"value": nw * 54 * steps / dt, "unit": UNIT, "kind": "reference", "cores": int(d["threads"]),
            "sample": f"{nw} walkers x {steps} VMC sweeps after 1 untimed, same trial function, "
                      "kinetic energy only (the reference has no 3-D Ewald)"}


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nw = min(a.walkers, a.cpu_walkers)
    v, info = run_reference_cpu(nw, a.steps, a.warmup, a.seed)
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "impl": "reference",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: seeded uniform initial walkers (mt19937_64)",
        "config": {"workload": WORKLOAD, "walkers": nw, "n_particles": NP, "rs": RS, "tau": TAU},
        "cpu_baseline": dict(value=v, unit=UNIT, **info),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ───────────────────────── GPU arm ──────────────────────────────────────

class DmcLoop:
    """Population control around dmc_advance/dmc_branch, the loop of
    DMC::run_one_step (src/qmc/dmc.cpp:693-739) with PopulationControl's
    trial-energy feedback (src/qmc/population_control.cpp:37-103)."""

    def __init__(self, walkers, target, seed):
        import alea_b200
        self.g = walkers
        self.target = target
        walkers.set_streams(seed, alea_b200.STREAM_DMC, target)
        self.state = branch_stream_state(seed)
        el = walkers.download()["local_energy"]
        self.etrial = self.eref = float(np.mean(el))
        med = np.median(el)
        sigma = 1.4826 * np.median(np.abs(el - med))
        self.e_cut = CUTOFF_ALPHA * np.sqrt(sigma * np.sqrt(NP) / TAU) if sigma > 0 else np.inf
        self.e_max = 1.5 * self.e_cut
        self.feedback = 1.0 / (GENERATIONS * TAU)

    def step(self):
        g = self.g
        st = g.dmc_advance(TAU, 1, self.etrial, self.eref, self.e_cut, self.e_max)
        ms = g.last_kernel_ms()
        g.dmc_branch(self.state, self.target)
        if st.weight_sum > 0:
            self.eref = st.energy_sum / st.weight_sum
            self.etrial = self.eref - self.feedback * np.log(st.weight_sum / self.target)
        return st, ms


def _splitmix64(x):
    m = (1 << 64) - 1
    x = (x + 0x9E3779B97F4A7C15) & m
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & m
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & m
    return x ^ (x >> 31)


def branch_stream_state(seed):
    """xoshiro256++ state of the serial branch stream, as alea_gpu_dmc_run
    seeds it: stream_seed(seed, "dmc-brch", 0) expanded by splitmix64."""
    import alea_b200
    base = _splitmix64(_splitmix64(_splitmix64(seed) ^ alea_b200.STREAM_BRANCH) ^ 0)
    m = (1 << 64) - 1
    return np.array([_splitmix64((base + i * 0x9E3779B97F4A7C15) & m) for i in range(4)],
                    dtype=np.uint64)


def gpu_arm(a):
    import torch
    import torch.distributed as dist

    import alea_b200
    from alea_b200 import _capi
    from alea_b200 import setup as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device; the walker path has no CPU fallback")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    from alea_b200.replicas import Replicas, replica_seed
    reps = Replicas(dist if world > 1 else None, dev)
    barrier = reps.barrier

    nw = a.walkers
    setup = S.heg2d(N_UP, N_DOWN, RS, PADE_B)
    desc = setup.desc
    b_move, b_eval, n_kj, n_ke = work_per_unit(desc)
    seed = replica_seed(a.seed, rank)
    g = alea_b200.Walkers(desc, capacity=2 * nw + 2, device=local)
    g.upload(setup.positions(seed, nw))
    # untimed VMC pre-equilibration from the uniform start
    if a.pre > 0:
        g.vmc_run(0, 1, a.pre, 1, VMC_TAU, nw, seed)
    loop = DmcLoop(g, nw, seed)
    for _ in range(a.warmup):
        loop.step()
    stream = torch.cuda.ExternalStream(g.stream_handle(), device=dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # ── device-resident timed region ──
    dev_uuid = None
    try:
        dev_uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(dev_uuid)
    l0 = g.launch_count()
    torch.cuda.synchronize()
    ev0.record(stream)
    moves = evals = 0
    sweep_ms = []
    sweep_walkers = []
    energies = []
    for _ in range(a.steps):
        st, ms = loop.step()
        moves += st.n_proposed
        evals += st.n_walkers
        sweep_ms.append(ms)
        sweep_walkers.append(st.n_walkers)
        energies.append(st.energy_sum / st.weight_sum)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = g.launch_count() - l0
    clk = clocks.stop()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ms_max = reps.max(ms)
    moves_all = reps.sum(float(moves))
    evals_all = reps.sum(float(evals))
    launches_all = reps.sum(float(launches))
    value = moves_all / (ms_max * 1e-3)

    # roofline of the sweep kernel (the dominant launch)
    hbm_peak, peak_kind = measured_peaks()
    t_sweep = float(np.sum(sweep_ms)) * 1e-3
    bytes_alg = moves * b_move + evals * b_eval
    achieved = bytes_alg / t_sweep / 1e9
    per_walker = profiled_traffic_per_walker()
    traffic = per_walker * float(np.mean(sweep_walkers)) if per_walker else None
    # the sweep's binding roof: FP64 CUDA-core throughput (measured FMA loop)
    fpm = profiled_fp64_flops_per_move()
    fp64_peak = ctypes.c_double(0.0)
    _capi.load().alea_gpu_measure_fp64_peak(local, ctypes.byref(fp64_peak))
    roof64 = None
    if fpm and fp64_peak.value > 0.0:
        ach64 = fpm * moves / t_sweep / 1e12
        roof64 = {"bound": "fp64", "achieved": ach64, "peak": fp64_peak.value, "unit": "TFLOP/s",
                  "frac": ach64 / fp64_peak.value, "flops_per_move": fpm,
                  "peak_kind": "measured: FP64 FMA loop on this GPU (alea_gpu_measure_fp64_peak)",
                  "kernel": "sweep_fast_kernel (one-warp DMC sweep)"}

    # ── the FP32 form on the same start: throughput and energy against FP64 ──
    fp32 = None
    if not a.no_fp32:
        f = alea_b200.Walkers(desc, capacity=2 * nw + 2, device=local)
        f.upload(setup.positions(seed, nw))
        f.set_precision("fp32")
        if a.pre > 0:
            f.vmc_run(0, 1, a.pre, 1, VMC_TAU, nw, seed)
        floop = DmcLoop(f, nw, seed)
        for _ in range(a.warmup):
            floop.step()
        fstream = torch.cuda.ExternalStream(f.stream_handle(), device=dev)
        torch.cuda.synchronize()
        barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(fstream)
        fmoves, fms, fen = 0, [], []
        for _ in range(a.steps):
            fst, fstep_ms = floop.step()
            fmoves += fst.n_proposed
            fms.append(fstep_ms)
            fen.append(fst.energy_sum / fst.weight_sum)
        f1.record(fstream)
        torch.cuda.synchronize()
        barrier()
        fms_max = reps.max(f0.elapsed_time(f1))
        fmoves_all = reps.sum(float(fmoves))
        e64, e32 = float(np.mean(energies)), float(np.mean(fen))
        err = float(np.sqrt(np.var(energies) / max(len(energies) - 1, 1) + np.var(fen) / max(len(fen) - 1, 1)))
        # paired: both walks start from the same walkers with the same random
        # streams, so step t of one follows step t of the other until accept
        # or branch decisions part them; the per-step differences carry the
        # bias with a far smaller scatter than either walk
        diff = np.array(fen) - np.array(energies)
        err_paired = float(np.std(diff, ddof=1) / np.sqrt(len(diff))) if len(diff) > 1 else None
        fp32 = {"value": fmoves_all / (fms_max * 1e-3), "unit": UNIT, "ms_per_step": fms_max / a.steps,
                "sweep_ms_per_launch": float(np.mean(fms)),
                "energy_per_particle": e32 / NP, "energy_per_particle_fp64": e64 / NP,
                "bias_per_particle": (e32 - e64) / NP, "bias_error_per_particle": err / NP,
                "bias_paired_error_per_particle": err_paired / NP if err_paired is not None else None,
                "ratio_to_fp64": (fmoves_all / (fms_max * 1e-3)) / value,
                "note": "FP32 and FP64 walks from the same walkers and random streams, mean of the timed "
                        "steps' mixed estimators; bias_error from the two walks' step-to-step scatter as if "
                        "independent, bias_paired_error from the scatter of the per-step differences"}
        f.close()

    # ── end to end through the C ABI from pinned host buffers ──
    lib = _capi.load()
    final = g.download()
    n_w = final["positions"].shape[0]
    pin_pos = torch.empty(NP * DIM * n_w, dtype=torch.float64, pin_memory=True)
    pin_pos.numpy()[:] = np.ascontiguousarray(final["positions"].T).ravel()
    pin_out = torch.empty(NP * DIM * (2 * nw + 2), dtype=torch.float64, pin_memory=True)
    pin_el = torch.empty(2 * nw + 2, dtype=torch.float64, pin_memory=True)
    cfg = _capi.RunConfig(0, 1, a.steps, 1, TAU, 1, nw, np.uint64(seed + 1).item(), nw,
                          GENERATIONS, CUTOFF_ALPHA)
    res = _capi.RunResult()
    dp = lambda t: ctypes_ptr(t, _capi)
    h0, d0 = g.transfer_bytes()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g._check(lib.alea_gpu_upload_walkers(g.ctx, dp(pin_pos), n_w))
    g._check(lib.alea_gpu_dmc_run(g.ctx, cfg, res, None))
    g._check(lib.alea_gpu_download_walkers(g.ctx, dp(pin_out), None, None, None, dp(pin_el), None))
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    h1, d1 = g.transfer_bytes()
    e_ms = reps.max(e0.elapsed_time(e1))
    e_moves = reps.sum(float(res.n_moves))
    e2e = {"value": e_moves / (e_ms * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": int((h1 - h0) / a.steps), "d2h_bytes_per_step": int((d1 - d0) / a.steps),
           "path": "alea_gpu_upload_walkers + alea_gpu_dmc_run + alea_gpu_download_walkers, pinned host buffers"}

    # ── device estimators on the same population: one measurement each step ──
    est = None
    if not a.no_estimators:
        av = np.array(desc["cell"]["vectors"], dtype=float).reshape(2, 2)
        ws = 0.5 * min(float(np.hypot(*(i * av[0] + j * av[1])))
                       for i in range(-2, 3) for j in range(-2, 3) if i or j)
        b1 = float(np.hypot(*(2.0 * np.pi * np.linalg.inv(av)[:, 0])))
        ids = [g.add_estimator("gofr", n_bins=110, rmax=ws),
               g.add_estimator("density", n_bins=48, rmax=ws, per_particle=a.density_per_particle),
               g.add_estimator("sofk", kmax=8.0 * b1)]
        g.estimators_accumulate()          # first measurement allocates the running blocks
        torch.cuda.synchronize()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l_est = g.launch_count()
        x0.record(stream)
        for _ in range(a.steps):
            g.estimators_accumulate()
        x1.record(stream)
        torch.cuda.synchronize()
        est_ms = x0.elapsed_time(x1) / a.steps
        est = {"ms_per_measurement": est_ms, "share_of_dmc_step": est_ms / (ms_max / a.steps),
               "launches_per_measurement": (g.launch_count() - l_est) / a.steps,
               "walkers": int(g.nw),
               "estimators": f"gofr 110 bins to r = {ws:.1f}, density 48x48 per "
                             f"{'particle' if a.density_per_particle else 'spin'}, "
                             f"sofk n_k = {g.estimator_desc(ids[2]).n_k} (|k| <= 8 |b1|)",
               "note": "every walker binned on the device; the host reads one block estimate per block"}
        g.clear_estimators()

    # ── the VMC benchmark (config 1): 512 walkers, 100 blocks x 50 sweeps ──
    vmc_c1 = None
    if a.vmc_blocks > 0:
        v = alea_b200.Walkers(desc, capacity=512, device=local)
        v.upload(setup.positions(seed + 7, 512))
        vstream = torch.cuda.ExternalStream(v.stream_handle(), device=dev)
        torch.cuda.synchronize()
        barrier()
        v0, v1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        v0.record(vstream)
        vres, _ = v.vmc_run(0, a.vmc_blocks, 10, 5, VMC_TAU, 8, seed + 8)
        v1.record(vstream)
        torch.cuda.synchronize()
        barrier()
        vms = reps.max(v0.elapsed_time(v1))
        vmc_c1 = {"value": reps.sum(float(vres.n_moves)) / (vms * 1e-3), "unit": UNIT,
                  "el_evals_per_s": reps.sum(float(vres.n_evaluations)) / (vms * 1e-3),
                  "walkers": 512, "blocks": a.vmc_blocks, "sweeps_per_block": 50,
                  "energy_per_particle": vres.energy / NP, "error_per_particle": vres.energy_error / NP,
                  "acceptance": vres.acceptance, "seconds": vms * 1e-3,
                  "note": "VMC of the same system, Metropolis step 0.5 rs, 8 random streams, from a uniform "
                          "start (no equilibration blocks: the first blocks are in the mean)"}
        v.close()

    # ── other trial functions of the same gas, VMC sweeps timed on the device ──
    def vmc_sweeps(d, pos, n_walkers, steps, tau):
        v = alea_b200.Walkers(d, capacity=n_walkers, device=local)
        v.upload(pos)
        v.set_streams(seed + 11, alea_b200.STREAM_VMC, n_walkers)
        vs = torch.cuda.ExternalStream(v.stream_handle(), device=dev)
        for _ in range(max(a.warmup, 3)):
            v.vmc_step(tau, 1, False)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(vs)
        acc = 0
        for _ in range(steps):
            acc += v.vmc_step(tau, 1, False).n_accepted
        e1.record(vs)
        torch.cuda.synchronize()
        barrier()
        t = reps.max(e0.elapsed_time(e1)) * 1e-3
        n = n_walkers * int(d["np"]) * steps
        out = {"value": reps.sum(float(n)) / t, "unit": UNIT, "walkers": n_walkers, "sweeps": steps,
               "ms_per_sweep": t * 1e3 / steps, "acceptance": acc / n,
               "energy_per_particle": float(np.mean(v.download()["local_energy"])) / int(d["np"])}
        v.close()
        return out

    others = None
    if a.other_systems:
        from alea_b200 import setup as S
        tw = S.heg2d_twisted(21, 21, RS, (0.125, 0.125))
        others = {
            "twisted_heg42": dict(vmc_sweeps(tw.desc, tw.positions(seed + 12, nw), nw, 5, VMC_TAU),
                                  sweep="one-warp complex sweep",
                                  system="N=42 rs=30 at twist (1/8, 1/8): complex determinant"),
            "backflow_heg42": dict(vmc_sweeps(S.with_backflow(desc), setup.positions(seed + 13, 2048), 2048, 3,
                                              VMC_TAU),
                                   sweep="generic CTA sweep, one pivoted Gauss-Jordan per determinant per move",
                                   system="N=42 rs=30 with backflow determinants (C=3, L at the inradius)"),
        }
        tw.close()
        # the fourth configuration: the 3-D backflow gas, 54 electrons at r_s = 5, 3-D Ewald, 4096 walkers
        g3 = S.heg3d(27, 27, 5.0)
        others["backflow_heg54_3d"] = dict(
            vmc_sweeps(g3.desc, g3.positions(seed + 14, 4096), 4096, 2, 1.0),
            sweep="3-D CTA sweep (alea_bf3d.cu), one warp Gauss-Jordan per spin determinant per move",
            system="3-D electron gas N=54 (27+27) rs=5, backflow determinants of plane waves (C=3, c0=0.1, "
                   "L = half the cell side), Drummond Jastrows, 3-D Ewald (%d k-vectors)" % len(g3.desc["ewald"]["weight"]))
        g3.close()
        c4 = others["backflow_heg54_3d"]
        if fp64_peak.value > 0.0:
            # the two spins' 27x27 inversions of every move, N^3 FMAs each, against the FP64 FMA peak
            f_move = 2 * 2 * 27 ** 3
            ach = c4["value"] * f_move * 1e-12
            c4["roofline_fp64"] = {"bound": "fp64", "achieved": ach, "peak": fp64_peak.value, "unit": "TFLOP/s",
                                   "frac": ach / fp64_peak.value, "flops_per_move": f_move,
                                   "note": "algorithmic: the move's two Gauss-Jordan inversions (2 x N^3 FMAs); "
                                           "refresh, orbitals and local energy not counted"}
        if rank == 0:
            c4["cpu_reference"] = reference_vmc_3d(256, 3, seed)

    # ── the serving mix through the packed server (config 5), rank 0 only ──
    serving = None
    if rank == 0 and world == 1 and a.serve_bench_jobs > 0:
        serving = run_serving(a, a.serve_bench_jobs, packed=True)
        unpacked = run_serving(a, a.serve_bench_jobs, packed=False)
        serving["unpacked"] = {k: unpacked[k] for k in ("value", "p50_ms", "p99_ms", "mean_queue_ms",
                                                        "mean_run_ms", "wall_s")}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            v, info = run_reference_cpu(min(nw, a.cpu_walkers), a.cpu_steps, 1, a.seed)
            cpu = dict(value=v, unit=UNIT, **info)
        except Exception as exc:   # reported, never substituted for the GPU number
            cpu = {"value": None, "unit": UNIT, "error": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: seeded uniform initial walkers (mt19937_64), VMC-equilibrated "
                    f"for {a.pre} steps; trial function and tables built on the host",
            "config": {"workload": WORKLOAD, "walkers": nw, "n_particles": NP, "rs": RS, "tau": TAU,
                       "pade": "u = a r/(1 + 0.3 r), a from the cusp: 1 (up-down), 1/3 (same spin)",
                       "ewald_k_vectors": n_ke, "jastrow_k_vectors": n_kj,
                       "l2": "no flush: walker records (~50 KB x walkers) exceed the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "el_evals_per_s": evals_all / (ms_max * 1e-3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "kernel": "sweep_fast_kernel (one-warp DMC sweep)", "peak_kind": peak_kind,
                         "bytes_per_move": b_move, "bytes_per_eval": b_eval,
                         "sweep_ms_per_launch": float(np.mean(sweep_ms)),
                         "sweep_share_of_step": t_sweep / (ms * 1e-3)},
            "roofline_fp64": roof64,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches_all),
            "clocks": clk,
            "population": int(g.nw),
            "fp32": fp32,
            "estimators": est,
            "serving": serving,
            "vmc_c1": vmc_c1,
            "other_systems": others,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ───────────────────────── serving mix ──────────────────────────────────

SERVE_SAMPLES = 1 << 20          # electron moves per job
SERVE_WALKERS = 1024
TWIST_GRID = [(i + 0.5) / 4.0 for i in range(4)]


def run_serving(a, n_jobs, packed=True, rate=None, slots=None):
    """The serving mix of the workload list: VMC jobs of 2^20 moves each,
    arriving Poisson at `rate`, half from the 2-D electron gas (N = 26, 42,
    58, 90 at rs = 30, 40, 60, each at one of the 4x4 offset twists that does
    not split a shell: complex determinants) and half from the 2-D dipolar
    bosons (N = 256, C/r^3, zero-energy Jastrow).  Every job goes through
    alea_gpu_submit_job / alea_gpu_poll on one server (packed: every admitted
    VMC job steps in the same sweep launches); latency is submission to
    completion.  Returns the summary dict."""
    import torch
    import alea_b200
    from alea_b200 import setup as S
    rate = a.serve_rate if rate is None else rate
    slots = a.serve_slots if slots is None else slots
    rng = np.random.default_rng(a.seed)
    heg = [(n, rs, (x, y)) for n in (13, 21, 29, 45) for rs in (30.0, 40.0, 60.0)
           for x in TWIST_GRID for y in TWIST_GRID]
    picks, setups = [], {}
    def setup_of(key):
        if key not in setups:
            try:
                setups[key] = (S.heg2d_twisted(key[1], key[1], key[2], key[3]) if key[0] == "heg"
                               else S.dipoles2d(256, 0.0353, 1.0, 3.0, 0.0459))
            except ValueError:       # this twist splits a shell at this N: not a valid job
                setups[key] = None
        return setups[key]

    while len(picks) < n_jobs:
        if rng.random() < 0.5:       # the family first, 50/50; then a valid member of it
            while True:
                n, rs, t = heg[rng.integers(len(heg))]
                key = ("heg", n, rs, t)
                if setup_of(key) is not None:
                    break
        else:
            key = ("dipoles", 256, 0.0353, None)
            setup_of(key)
        picks.append(key)
    jobs = []
    for i, key in enumerate(picks):
        kind, n, rs, t = key
        st = setups[key]
        np_tot = st.desc["np"]
        sweeps = -(-SERVE_SAMPLES // (SERVE_WALKERS * np_tot))
        n_acc = 4
        steps = -(-sweeps // (n_acc + 1))
        tau = (0.5 * rs) ** 2 if kind == "heg" else 0.0003
        pos = st.positions(a.seed + i, SERVE_WALKERS)
        jobs.append((st, pos, steps, n_acc, tau, key))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(jobs)))
    srv = alea_b200.Server(max_running=slots, packed=packed)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = []
    for (st, pos, steps, n_acc, tau, key), t_arr in zip(jobs, arrivals):
        delay = t0 + t_arr - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        ids.append(srv.submit(st.desc, pos, 0, 1, n_acc, steps, 1, tau, seed=a.seed + len(ids)))
    results = [srv.poll(i, timeout_ms=600000) for i in ids]
    wall = time.perf_counter() - t0
    srv.close()
    ok = [r for r in results if r is not None and r.status == 0]
    lat = np.array([r.latency_ms for r in ok])
    moves = float(sum(r.result.n_moves for r in ok))
    kinds = {}
    for (st, pos, steps, n_acc, tau, key), r in zip(jobs, results):
        label = f"heg N={2 * key[1]} rs={key[2]:g}" if key[0] == "heg" else "dipoles N=256"
        kinds.setdefault(label, []).append(r.latency_ms if r is not None else None)
    return {
        "value": moves / wall, "unit": "moves/s",
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_queue_ms": float(np.mean([r.queue_ms for r in ok])) if ok else None,
        "mean_run_ms": float(np.mean([r.run_ms for r in ok])) if ok else None,
        "requested_moves_per_s": float(rate * SERVE_SAMPLES),
        "jobs": len(jobs), "completed": len(ok), "wall_s": wall, "arrival_rate_per_s": rate,
        "dipole_jobs": sum(1 for k in picks if k[0] == "dipoles"),
        "packed": bool(packed), "slots": slots,
        "latency_by_kind_ms": {k: float(np.median([x for x in v if x is not None])) for k, v in kinds.items()},
    }


def serve_arm(a):
    """--serve: the serving mix alone, one JSON line."""
    import torch
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: no CUDA device")
    r = run_serving(a, a.serve_jobs, packed=not a.serve_unpacked)
    line = {
        "metric": "serving: aggregate electron-moves/s, p50/p99 job latency", "value": r.pop("value"),
        "unit": r.pop("unit"), "n_gpus": 1, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic: seeded uniform walkers per job, Poisson arrivals",
        "config": {"workload": "serving mix: VMC jobs of 2^20 moves, 1024 walkers; half 2-D electron gas "
                               "N in {26,42,58,90} x rs in {30,40,60} x 4x4 offset twists (complex), "
                               "half 2-D dipolar bosons N=256",
                   "jobs": r["jobs"], "arrival_rate_per_s": r["arrival_rate_per_s"], "slots": r["slots"],
                   "packed": r["packed"]},
    }
    line.update(r)
    print(json.dumps(line), flush=True)
    return 0


def ctypes_ptr(t, _capi):
    import ctypes
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), _capi.c_dp)


def main():
    a = parse()
    if a.impl == "reference":
        return reference_arm(a)
    if a.serve:
        return serve_arm(a)
    return gpu_arm(a)


if __name__ == "__main__":
    sys.exit(main())
