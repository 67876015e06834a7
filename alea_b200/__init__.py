"""alea_b200 — B200-native VMC/DMC walker hot path for Alea.

The walker ensemble lives in HBM; every sweep, local energy and branching
gather runs in the sm_100a kernels of ``libalea_b200.so`` behind the C ABI of
``include/alea_gpu.h``.  This module is the thin Python view of that ABI used
by tests and the benchmark; C/C++ hosts call the ABI directly.

A system is described by a plain dict (the schema of ``setup.describe_*``,
see ``alea_b200/setup.py``): cell, particle groups, determinant blocks with
their orbitals, pair Jastrows (Padé with image-sum tables, Drummond), Ewald
tables and open Coulomb terms.
"""
from __future__ import annotations

import ctypes
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from . import _capi
from . import estimators as _est
from ._capi import load as _load

__all__ = ["Walkers", "Server", "AleaGpuError", "pack_system", "STREAM_VMC", "STREAM_DMC", "STREAM_BRANCH"]

STREAM_VMC = _capi.STREAM_VMC
STREAM_DMC = _capi.STREAM_DMC
STREAM_BRANCH = _capi.STREAM_BRANCH


class AleaGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"alea_gpu error {code} ({_capi.ERRORS.get(code, '?')}): {msg}")
        self.code = code


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_capi.c_dp)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_capi.c_ip)


def pack_system(desc: Dict[str, Any]):
    """alea_gpu_system from a description dict.  Returns (struct, keepalive)."""
    keep: List[np.ndarray] = []

    def f64(x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        keep.append(a)
        return a

    def i32(x):
        a = np.ascontiguousarray(np.asarray(x, dtype=np.int32))
        keep.append(a)
        return a

    s = _capi.System()
    s.dim = int(desc["dim"])
    s.n_particles = int(desc["np"])
    cell = desc["cell"]
    s.periodic = int(cell["periodic"])
    if s.periodic:
        for i, v in enumerate(cell["vectors"]):
            s.lattice[i] = float(v)
    groups = desc["groups"]
    s.n_groups = len(groups)
    for i, g in enumerate(groups):
        G = s.groups[i]
        G.first, G.last, G.charge = int(g["first"]), int(g["last"]), float(g["charge"])
        for d, v in enumerate(g["inv_mass"]):
            G.inv_mass[d] = float(v)
    blocks = desc.get("slater", [])
    s.n_blocks = len(blocks)
    for i, b in enumerate(blocks):
        B = s.blocks[i]
        B.first, B.last = int(b["first"]), int(b["last"])
        if b["type"] == "twisted_plane_wave":
            B.type = _capi.ORB_TWISTED_PLANE_WAVE
            B.k = _dp(f64(b["q"]))
        elif b["type"] == "plane_wave":
            B.type = _capi.ORB_PLANE_WAVE
            B.k = _dp(f64(b["k"]))
            B.is_sin = _ip(i32(b["is_sin"]))
        else:
            B.type = _capi.ORB_GAUSSIAN
            B.centers = _dp(f64(b["centers"]))
            B.alphas = _dp(f64(b["alphas"]))
            B.opt_alpha = int(b.get("opt_alpha", 0))
    terms = []
    for p in desc.get("pade", []):
        terms.append(("pade", p))
    for d in desc.get("drummond", []):
        terms.append(("drummond", d))
    for z in desc.get("zero_energy", []):
        terms.append(("zero_energy", z))
    s.n_terms = len(terms)
    for i, (kind, t) in enumerate(terms):
        T = s.terms[i]
        if kind == "pade":
            T.kind = _capi.PAIR_PADE
            T.n_pairs = 1
            pr = [int(t["ga"][0]), int(t["ga"][1]), int(t["gb"][0]), int(t["gb"][1])]
            for k in range(4):
                T.pairs[0][k] = pr[k]
            a, b = list(t["a"]), list(t["b"])
            T.num_order, T.den_order = len(a), len(b)
            for k, v in enumerate(a + b):
                T.coeffs[k] = float(v)
            im = t.get("image_sum")
            T.image_sum = 1 if im else 0
            if im:
                sp = im["spline"]
                T.short_range.r_cut = float(sp["r_cut"])
                T.short_range.inv_delta = float(sp["inv_delta"])
                T.short_range.n_knots = int(sp["n_knots"])
                T.short_range.scaled = _dp(f64(sp["scaled"]))
                T.u_inf = float(im["u_inf"])
                T.kset.n_k = len(im["weight"])
                T.kset.n1 = _ip(i32(im["n1"]))
                T.kset.n2 = _ip(i32(im["n2"]))
                T.kset.kx = _dp(f64(im["kx"]))
                T.kset.ky = _dp(f64(im["ky"]))
                T.kset.weight = _dp(f64(im["weight"]))
            opts = t.get("opt", [])
            T.n_opt = len(opts)
            for q, o in enumerate(opts):
                T.opt_index[q] = int(o["index"])
                if im:
                    T.opt_inf[q] = float(o["inf"])
                    sp = o["spline"]
                    S = T.opt_short_range[q]
                    S.r_cut, S.inv_delta, S.n_knots = float(sp["r_cut"]), float(sp["inv_delta"]), int(sp["n_knots"])
                    S.scaled = _dp(f64(sp["scaled"]))
                    T.opt_weight[q] = _dp(f64(o["weight"]))
        elif kind == "zero_energy":
            T.kind = _capi.PAIR_ZERO_ENERGY
            T.n_pairs = 1
            pr = [int(t["ga"][0]), int(t["ga"][1]), int(t["gb"][0]), int(t["gb"][1])]
            for k in range(4):
                T.pairs[0][k] = pr[k]
            T.ze_b = float(t["b"])
            T.ze_exponent = float(t["exponent"])
            T.ze_matching_radius = float(t["matching_radius"])
            T.ze_cutoff = float(t["cutoff"])
        else:
            T.kind = _capi.PAIR_DRUMMOND
            T.n_pairs = len(t["pairs"])
            for q, pr in enumerate(t["pairs"]):
                for k in range(4):
                    T.pairs[q][k] = int(pr[k])
            T.C = int(t["C"])
            T.gamma = float(t["gamma"])
            T.L = float(t["L"])
            T.n_coeffs = len(t["coeffs"])
            for k, v in enumerate(t["coeffs"]):
                T.dcoeffs[k] = float(v)
            opts = t.get("opt", [])
            T.n_opt = len(opts)
            for q, o in enumerate(opts):
                T.opt_index[q] = int(o["index"])
    ew = desc.get("ewald")
    if ew:
        E = s.ewald
        E.enabled = 1
        E.r_cut = float(ew["r_cut"])
        E.inv_eps = float(ew.get("inv_eps", 1.0))
        E.constant = float(ew["self_energy"]) + float(ew.get("background_energy", 0.0))
        sp = ew["spline"]
        E.long_range.r_cut = float(sp["r_cut"])
        E.long_range.inv_delta = float(sp["inv_delta"])
        E.long_range.n_knots = int(sp["n_knots"])
        E.long_range.scaled = _dp(f64(sp["scaled"]))
        E.kset.n_k = len(ew["weight"])
        E.kset.n1 = _ip(i32(ew["n1"]))
        E.kset.n2 = _ip(i32(ew["n2"]))
        E.kset.kx = _dp(f64(ew["kx"]))
        E.kset.ky = _dp(f64(ew["ky"]))
        E.kset.weight = _dp(f64(ew["weight"]))
        if "kz" in ew:   # a 3-D cell
            E.kset.n3 = _ip(i32(ew["n3"]))
            E.kset.kz = _dp(f64(ew["kz"]))
    cl = desc.get("coulomb", [])
    s.n_coulomb = len(cl)
    for i, c in enumerate(cl):
        C = s.coulomb[i]
        C.a_first, C.a_last = int(c["ga"][0]), int(c["ga"][1])
        C.b_first, C.b_last = int(c["gb"][0]), int(c["gb"][1])
        C.coef = float(c["coef"])
    ip = desc.get("inverse_power", [])
    s.n_inverse_power = len(ip)
    for i, c in enumerate(ip):
        V = s.inverse_power[i]
        V.a_first, V.a_last = int(c["ga"][0]), int(c["ga"][1])
        V.b_first, V.b_last = int(c["gb"][0]), int(c["gb"][1])
        V.strength, V.exponent, V.tail = float(c["strength"]), float(c["exponent"]), float(c["tail"])
    bf = desc.get("backflow", [])
    s.n_backflow = len(bf)
    for i, b in enumerate(bf):
        F = s.backflow[i]
        F.first, F.last = int(b["first"]), int(b["last"])
        if b["type"] == "plane_wave":
            F.type = _capi.ORB_PLANE_WAVE
            F.k = _dp(f64(b["k"]))
            F.is_sin = _ip(i32(b["is_sin"]))
        else:
            F.type = _capi.ORB_GAUSSIAN
            F.centers = _dp(f64(b["centers"]))
            F.alphas = _dp(f64(b["alphas"]))
        F.n_channels = len(b["channels"])
        for q, ch in enumerate(b["channels"]):
            C = F.channels[q]
            C.source_first, C.source_last = int(ch["source_first"]), int(ch["source_last"])
            C.C, C.L = int(ch["C"]), float(ch["L"])
            C.n_coeffs = len(ch["coeffs"])
            for k, v in enumerate(ch["coeffs"]):
                C.coeffs[k] = float(v)
            C.zero_slope = int(ch.get("zero_slope", 0))
            opt = ch.get("opt_index", [])
            C.n_opt = len(opt)
            for q, v in enumerate(opt):
                C.opt_index[q] = int(v)
    return s, keep


class Walkers:
    """A context on one device holding up to ``capacity`` walkers of a system."""

    def __init__(self, desc: Dict[str, Any], capacity: int, device: int = 0):
        self.lib = _load()
        self.desc = desc
        self.np = int(desc["np"])
        self.dim = int(desc["dim"])
        sysc, keep = pack_system(desc)
        ctx = ctypes.c_void_p()
        rc = self.lib.alea_gpu_create(ctypes.byref(sysc), device, int(capacity), ctypes.byref(ctx))
        if rc != 0:
            raise AleaGpuError(rc, self.lib.alea_gpu_last_error(None).decode())
        self.ctx = ctx
        self.capacity = int(capacity)

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.alea_gpu_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, precision: str) -> None:
        """'fp64' (the drop-in) or 'fp32' (the FP32 form of the sweeps)."""
        code = {"fp64": _capi.PRECISION_FP64, "fp32": _capi.PRECISION_FP32}[precision]
        self._check(self.lib.alea_gpu_set_precision(self.ctx, code))

    def _check(self, rc: int):
        if rc != 0:
            raise AleaGpuError(rc, self.lib.alea_gpu_last_error(self.ctx).decode())

    @property
    def nw(self) -> int:
        n = ctypes.c_int()
        self._check(self.lib.alea_gpu_num_walkers(self.ctx, ctypes.byref(n)))
        return n.value

    def upload(self, positions_aos: np.ndarray) -> None:
        """Walkers from AoS positions [w][p][d]; evaluates ψ and E_L."""
        pos = np.asarray(positions_aos, dtype=np.float64).reshape(-1, self.np * self.dim)
        nw = pos.shape[0]
        soa = np.ascontiguousarray(pos.T)   # [p*dim + d][w]
        self._check(self.lib.alea_gpu_upload_walkers(self.ctx, _dp(soa), nw))

    def evaluate(self) -> None:
        self._check(self.lib.alea_gpu_evaluate(self.ctx))

    def measure(self) -> None:
        self._check(self.lib.alea_gpu_measure(self.ctx))

    def download(self) -> Dict[str, np.ndarray]:
        nw = self.nw
        n = self.np * self.dim
        pos = np.zeros(n * nw)
        grad = np.zeros(n * nw)
        lap = np.zeros(n * nw)
        lp = np.zeros(nw)
        el = np.zeros(nw)
        w = np.zeros(nw)
        self._check(self.lib.alea_gpu_download_walkers(self.ctx, _dp(pos), _dp(lp), _dp(grad),
                                                       _dp(lap), _dp(el), _dp(w)))
        return {
            "positions": pos.reshape(n, nw).T.copy(),
            "grad": grad.reshape(n, nw).T.copy(),
            "lap": lap.reshape(n, nw).T.copy(),
            "log_psi": lp, "local_energy": el, "weights": w,
        }

    def download_phase(self) -> Dict[str, np.ndarray]:
        """Phase planes and Im E_L of a complex (twisted) trial function."""
        nw = self.nw
        n = self.np * self.dim
        pg = np.zeros(n * nw)
        pl = np.zeros(n * nw)
        eli = np.zeros(nw)
        self._check(self.lib.alea_gpu_download_phase(self.ctx, _dp(pg), _dp(pl), _dp(eli)))
        return {"phase_grad": pg.reshape(n, nw).T.copy(), "phase_lap": pl.reshape(n, nw).T.copy(),
                "local_energy_imag": eli}

    def move(self, p: int, new_pos_aos: np.ndarray, accept: Optional[Sequence[bool]] = None):
        """Single-particle move of p for every walker; new_pos_aos [w][d]."""
        nw = self.nw
        npos = np.ascontiguousarray(np.asarray(new_pos_aos, dtype=np.float64).reshape(nw, self.dim).T)
        lr = np.zeros(nw)
        ph = np.zeros(nw)
        ng = np.zeros(self.dim * nw)
        nl = np.zeros(self.dim * nw)
        if accept is not None:
            mask = np.ascontiguousarray(np.asarray(accept, dtype=np.uint8))
            mp = mask.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))
        else:
            mp = None
        self._check(self.lib.alea_gpu_move(self.ctx, int(p), _dp(npos), mp, _dp(lr), _dp(ph),
                                           _dp(ng), _dp(nl)))
        return lr, ph, ng.reshape(self.dim, nw).T, nl.reshape(self.dim, nw).T

    def set_streams(self, seed: int, kind: int, n: int) -> None:
        self._check(self.lib.alea_gpu_set_streams(self.ctx, ctypes.c_uint64(seed),
                                                  ctypes.c_uint64(kind), int(n)))

    def vmc_step(self, tau: float, n_substeps: int = 1, drift: bool = False) -> _capi.StepStats:
        prm = _capi.VmcParams(tau, n_substeps, 1 if drift else 0)
        st = _capi.StepStats()
        self._check(self.lib.alea_gpu_vmc_step(self.ctx, ctypes.byref(prm), ctypes.byref(st)))
        return st

    def vmc_step_noalloc(self, tau: float, n_substeps: int = 1, drift: bool = False) -> _capi.StepStats:
        """alea_gpu_vmc_step_noalloc: the VMC step with its scratch in a static device array."""
        prm = _capi.VmcParams(tau, n_substeps, 1 if drift else 0)
        st = _capi.StepStats()
        self._check(self.lib.alea_gpu_vmc_step_noalloc(self.ctx, ctypes.byref(prm), ctypes.byref(st)))
        return st

    def dmc_advance(self, tau, n_substeps, e_trial, e_ref, e_cut, e_max) -> _capi.StepStats:
        prm = _capi.DmcParams(tau, n_substeps, e_trial, e_ref, e_cut, e_max)
        st = _capi.StepStats()
        self._check(self.lib.alea_gpu_dmc_advance(self.ctx, ctypes.byref(prm), ctypes.byref(st)))
        return st

    def dmc_branch(self, state: np.ndarray, target: int) -> None:
        st = np.ascontiguousarray(state, dtype=np.uint64)
        self._check(self.lib.alea_gpu_dmc_branch(self.ctx, st.ctypes.data_as(
            ctypes.POINTER(ctypes.c_uint64)), int(target)))
        state[:] = st

    def stream_handle(self) -> int:
        """The cudaStream_t (as an int) the context's work is ordered on."""
        v = ctypes.c_void_p()
        self._check(self.lib.alea_gpu_stream(self.ctx, ctypes.byref(v)))
        return int(v.value or 0)

    def transfer_bytes(self):
        """(host->device, device->host) bytes copied by this context so far."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        self._check(self.lib.alea_gpu_transfer_bytes(self.ctx, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def launch_count(self) -> int:
        """Kernels launched by this context so far."""
        v = ctypes.c_uint64()
        self._check(self.lib.alea_gpu_launch_count(self.ctx, ctypes.byref(v)))
        return v.value

    def last_kernel_ms(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.alea_gpu_last_kernel_ms(self.ctx, ctypes.byref(v)))
        return v.value

    # ── configurations and carry-over ─────────────────────────────────────
    def final_configurations(self) -> np.ndarray:
        """AoS rows [w][p][d] of the current walkers (the checkpoint rows)."""
        n = ctypes.c_int()
        self._check(self.lib.alea_gpu_final_configurations(self.ctx, None, ctypes.byref(n)))
        rows = np.zeros(max(n.value, 1) * self.np * self.dim)
        self._check(self.lib.alea_gpu_final_configurations(self.ctx, _dp(rows), ctypes.byref(n)))
        return rows[:n.value * self.np * self.dim].reshape(n.value, self.np, self.dim)

    def seed_walker_rows(self, rows: np.ndarray, nw: int) -> None:
        """nw walkers from AoS rows, walker w taking row w mod len(rows)."""
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.float64).reshape(-1, self.np * self.dim))
        self._check(self.lib.alea_gpu_seed_walker_rows(self.ctx, _dp(r), r.shape[0], int(nw)))

    def set_checkpoint_hook(self, fn) -> None:
        """fn(walkers, tag, blocks_done) at dmc_run's milestones ("eq", "a25",
        "a50", "a75"); it may read self.final_configurations().  None: off."""
        if fn is None:
            self._ckpt = None
            self._check(self.lib.alea_gpu_set_checkpoint_hook(self.ctx, _capi.CHECKPOINT_FN(), None))
            return
        def hook(_user, _ctx, tag, done):
            fn(self, tag.decode(), int(done))
        self._ckpt = _capi.CHECKPOINT_FN(hook)   # kept alive with the context
        self._check(self.lib.alea_gpu_set_checkpoint_hook(self.ctx, self._ckpt, None))

    def carry_over(self, source: "Walkers", nw: int, keep_state: bool = False) -> None:
        """Seed this context from `source`'s walkers on the device: positions
        and a full evaluation, or (keep_state, same system) whole records."""
        mode = _capi.CARRY_STATE if keep_state else _capi.CARRY_POSITIONS
        self._check(self.lib.alea_gpu_carry_over(source.ctx, self.ctx, int(nw), mode))

    # ── estimators (include/alea_gpu.h, estimators) ────────────────────────
    def add_estimator(self, kind: str, n_bins: int = 0, rmax: float = 0.0, per_particle: bool = False,
                      kmax: float = 0.0) -> int:
        """'gofr' (rmax, n_bins), 'density' (n_bins, rmax for an open cell,
        per_particle) or 'sofk' (kmax); returns the estimator's id."""
        spec = _capi.EstimatorSpec(_est.KINDS[kind], int(n_bins), float(rmax), 1 if per_particle else 0,
                                   float(kmax))
        i = ctypes.c_int()
        self._check(self.lib.alea_gpu_add_estimator(self.ctx, ctypes.byref(spec), ctypes.byref(i)))
        self._est_specs = getattr(self, "_est_specs", {})
        self._est_specs[i.value] = dict(kind=kind, n_bins=int(n_bins), rmax=float(rmax),
                                        per_particle=bool(per_particle), kmax=float(kmax))
        return i.value

    def clear_estimators(self) -> None:
        self._check(self.lib.alea_gpu_clear_estimators(self.ctx))
        self._est_specs = {}

    def estimators_reset(self) -> None:
        self._check(self.lib.alea_gpu_estimators_reset(self.ctx))

    def estimators_start_block(self) -> None:
        self._check(self.lib.alea_gpu_estimators_start_block(self.ctx))

    def estimators_accumulate(self, weights: Optional[np.ndarray] = None, chains: int = 1) -> None:
        """One measurement; weights [nw] (None: the walkers' own)."""
        wp = None
        if weights is not None:
            w = np.ascontiguousarray(weights, dtype=np.float64)
            wp = _dp(w)
        self._check(self.lib.alea_gpu_estimators_accumulate(self.ctx, wp, int(chains)))

    def estimators_stop_block(self) -> None:
        self._check(self.lib.alea_gpu_estimators_stop_block(self.ctx))

    def estimator_desc(self, i: int) -> _capi.EstimatorDesc:
        d = _capi.EstimatorDesc()
        self._check(self.lib.alea_gpu_estimator_info(self.ctx, int(i), ctypes.byref(d)))
        return d

    def estimator_blocks(self, i: int) -> np.ndarray:
        """Block estimates [n_chains][n_blocks][block_width]."""
        d = self.estimator_desc(i)
        out = np.zeros(max(d.n_chains * d.n_blocks * d.block_width, 1))
        self._check(self.lib.alea_gpu_estimator_blocks(self.ctx, int(i), _dp(out)))
        return out[:d.n_chains * d.n_blocks * d.block_width].reshape(d.n_chains, d.n_blocks, d.block_width)

    def estimator_kvectors(self, i: int) -> Dict[str, np.ndarray]:
        d = self.estimator_desc(i)
        nk, ns = d.n_k, d.n_shells
        n1, n2, sh, cnt = (np.zeros(nk, np.int32), np.zeros(nk, np.int32), np.zeros(nk, np.int32),
                           np.zeros(ns, np.int32))
        kx, ky, sk = np.zeros(nk), np.zeros(nk), np.zeros(ns)
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(self.lib.alea_gpu_estimator_kvectors(
            self.ctx, int(i), n1.ctypes.data_as(ip), n2.ctypes.data_as(ip), _dp(kx), _dp(ky),
            sh.ctypes.data_as(ip), _dp(sk), cnt.ctypes.data_as(ip)))
        return dict(n1=n1, n2=n2, kx=kx, ky=ky, shell_of=sh, shell_k=sk, shell_count=cnt)

    def estimator_results(self, i: int) -> Dict[str, np.ndarray]:
        """The estimator's named series (the reference's finalize())."""
        spec = self._est_specs[i]
        groups = self.desc["groups"]
        d = self.estimator_desc(i)
        chains = self.estimator_blocks(i)
        flat = chains.reshape(-1, d.block_width)
        if spec["kind"] == "gofr":
            return _est.finalize_gofr(flat, groups, spec["rmax"], spec["n_bins"], d.volume)
        if spec["kind"] == "density":
            return _est.finalize_density(chains, groups, spec["n_bins"], spec["per_particle"])
        return _est.finalize_sofk(flat, groups, self.estimator_kvectors(i))

    # ── forward walking (pure estimators of a DMC run) ─────────────────────
    def parameter_derivatives(self) -> np.ndarray:
        """O_k = d ln psi / d p_k of the pair terms' optimisable parameters,
        [n_params][nw]."""
        n = ctypes.c_int()
        self._check(self.lib.alea_gpu_parameter_derivatives(self.ctx, None, ctypes.byref(n)))
        nw = self.nw
        out = np.zeros(max(n.value * nw, 1))
        self._check(self.lib.alea_gpu_parameter_derivatives(self.ctx, _dp(out), ctypes.byref(n)))
        return out[:n.value * nw].reshape(n.value, nw)

    def parameter_gradient_derivatives(self):
        """(dgrad, dlap), each [n_params][np*dim][nw]: the parameters'
        derivatives of grad ln psi and of the per-dimension Laplacians."""
        n = ctypes.c_int()
        self._check(self.lib.alea_gpu_parameter_gradient_derivatives(self.ctx, None, None, ctypes.byref(n)))
        nw, m = self.nw, self.np * self.dim
        g, l = np.zeros(max(n.value * m * nw, 1)), np.zeros(max(n.value * m * nw, 1))
        self._check(self.lib.alea_gpu_parameter_gradient_derivatives(self.ctx, _dp(g), _dp(l), ctypes.byref(n)))
        k = n.value * m * nw
        return g[:k].reshape(n.value, m, nw), l[:k].reshape(n.value, m, nw)

    def set_forward_walking(self, lags: Sequence[float], interval: int = 1) -> None:
        """Lags in imaginary time (strictly increasing; empty: off)."""
        a = np.ascontiguousarray(np.asarray(lags, dtype=np.float64))
        self._check(self.lib.alea_gpu_set_forward_walking(self.ctx, _dp(a) if a.size else None, int(a.size),
                                                          int(interval)))
        self._fw_specs = {i: {} for i in range(a.size)}

    def add_fw_estimator(self, lag: int, kind: str, n_bins: int = 0, rmax: float = 0.0,
                         per_particle: bool = False, kmax: float = 0.0) -> int:
        spec = _capi.EstimatorSpec(_est.KINDS[kind], int(n_bins), float(rmax), 1 if per_particle else 0,
                                   float(kmax))
        i = ctypes.c_int()
        self._check(self.lib.alea_gpu_add_fw_estimator(self.ctx, int(lag), ctypes.byref(spec), ctypes.byref(i)))
        self._fw_specs[int(lag)][i.value] = dict(kind=kind, n_bins=int(n_bins), rmax=float(rmax),
                                                 per_particle=bool(per_particle), kmax=float(kmax))
        return i.value

    def fw_result(self, lag: int) -> Dict[str, Any]:
        """Pure potential energy of lag index `lag`: summary and block values."""
        out = _capi.FwSummary()
        self._check(self.lib.alea_gpu_fw_result(self.ctx, int(lag), ctypes.byref(out), None))
        blocks = np.zeros(max(out.n_blocks, 1))
        self._check(self.lib.alea_gpu_fw_result(self.ctx, int(lag), ctypes.byref(out), _dp(blocks)))
        return dict(lag_time=out.lag_time, lag_steps=out.lag_steps, measurements=out.measurements,
                    surviving_fraction=out.surviving_fraction, potential=out.potential,
                    potential_error=out.potential_error, block_potentials=blocks[:out.n_blocks])

    def fw_estimator_results(self, lag: int, i: int) -> Dict[str, np.ndarray]:
        """Series of a pure estimator, keys labelled fw<lag> as the reference's
        forward-walking builders label them (gofr_fw0_up_down, ...)."""
        spec = self._fw_specs[int(lag)][i]
        d = _capi.EstimatorDesc()
        self._check(self.lib.alea_gpu_fw_estimator_info(self.ctx, int(lag), int(i), ctypes.byref(d)))
        out = np.zeros(max(d.n_chains * d.n_blocks * d.block_width, 1))
        self._check(self.lib.alea_gpu_fw_estimator_blocks(self.ctx, int(lag), int(i), _dp(out)))
        chains = out[:d.n_chains * d.n_blocks * d.block_width].reshape(d.n_chains, d.n_blocks, d.block_width)
        groups = self.desc["groups"]
        flat = chains.reshape(-1, d.block_width)
        if spec["kind"] == "gofr":
            res = _est.finalize_gofr(flat, groups, spec["rmax"], spec["n_bins"], d.volume)
        elif spec["kind"] == "density":
            res = _est.finalize_density(chains, groups, spec["n_bins"], spec["per_particle"])
        else:
            nk, ns = d.n_k, d.n_shells
            n1, n2, sh, cnt = (np.zeros(nk, np.int32), np.zeros(nk, np.int32), np.zeros(nk, np.int32),
                               np.zeros(ns, np.int32))
            kx, ky, sk = np.zeros(nk), np.zeros(nk), np.zeros(ns)
            ip = ctypes.POINTER(ctypes.c_int)
            self._check(self.lib.alea_gpu_fw_estimator_kvectors(
                self.ctx, int(lag), int(i), n1.ctypes.data_as(ip), n2.ctypes.data_as(ip), _dp(kx), _dp(ky),
                sh.ctypes.data_as(ip), _dp(sk), cnt.ctypes.data_as(ip)))
            res = _est.finalize_sofk(flat, groups, dict(n1=n1, n2=n2, kx=kx, ky=ky, shell_of=sh, shell_k=sk,
                                                        shell_count=cnt))
        return _est.relabel(res, f"fw{int(lag)}")

    def _run(self, fn, n_eq, n_acc, n_steps, n_substeps, tau, streams, seed, drift=False,
             target=0, generations=10.0, alpha=2.0, n_blocks_out=0):
        cfg = _capi.RunConfig(n_eq, n_acc, n_steps, n_substeps, tau, 1 if drift else 0, streams,
                              ctypes.c_uint64(seed), target, generations, alpha)
        res = _capi.RunResult()
        blocks = np.zeros(max(n_blocks_out, 1))
        self._check(fn(self.ctx, ctypes.byref(cfg), ctypes.byref(res), _dp(blocks)))
        return res, blocks[:n_blocks_out]

    def vmc_run(self, n_eq, n_acc, n_steps, n_substeps, tau, streams, seed, drift=False):
        T = min(streams, self.nw)
        return self._run(self.lib.alea_gpu_vmc_run, n_eq, n_acc, n_steps, n_substeps, tau, streams,
                         seed, drift=drift, n_blocks_out=T * n_acc)

    def dmc_run(self, n_eq, n_acc, n_steps, n_substeps, tau, streams, seed, target=0,
                generations=10.0):
        return self._run(self.lib.alea_gpu_dmc_run, n_eq, n_acc, n_steps, n_substeps, tau,
                         streams, seed, target=target, generations=generations, n_blocks_out=n_acc)


def vmc_run_packed(walkers: Sequence["Walkers"], runs: Sequence[Dict[str, Any]]):
    """alea_gpu_vmc_run_packed: the VMC runs of several contexts, every step
    one packed sweep launch for all of them.  runs[i] holds vmc_run's
    arguments for walkers[i] (n_eq, n_acc, n_steps, n_substeps, tau, streams,
    seed, drift).  Returns [(RunResult, status)]."""
    lib = _load()
    n = len(walkers)
    ctxs = (ctypes.c_void_p * n)(*[w.ctx for w in walkers])
    cfgs = (_capi.RunConfig * n)()
    for i, r in enumerate(runs):
        cfgs[i] = _capi.RunConfig(r["n_eq"], r["n_acc"], r["n_steps"], r["n_substeps"], r["tau"],
                                  1 if r.get("drift") else 0, r["streams"], ctypes.c_uint64(r["seed"]), 0,
                                  10.0, 2.0)
    res = (_capi.RunResult * n)()
    st = (ctypes.c_int * n)()
    rc = lib.alea_gpu_vmc_run_packed(ctxs, n, cfgs, res, st)
    if rc != 0:
        raise AleaGpuError(rc, lib.alea_gpu_last_error(None).decode())
    return [(res[i], st[i]) for i in range(n)]


class Server:
    """Serving front end over alea_gpu_server (include/alea_gpu.h, serving):
    jobs are queued, admitted by device-memory footprint and run
    ``max_running`` at a time, each on its own context and stream (packed:
    VMC jobs step together in packed launches, alea_gpu_server_create_packed).  The
    packed system tables and positions of a job are kept alive here until
    the job has finished."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, max_running: int = 8, packed: bool = False):
        self.lib = _load()
        h = ctypes.c_void_p()
        create = self.lib.alea_gpu_server_create_packed if packed else self.lib.alea_gpu_server_create
        rc = create(device, int(hbm_budget_bytes), int(max_running), ctypes.byref(h))
        if rc != 0:
            raise AleaGpuError(rc, "alea_gpu_server_create failed")
        self.h = h
        self._keep: Dict[int, Any] = {}

    def submit(self, desc: Dict[str, Any], positions_aos: np.ndarray, mode: int, n_eq: int, n_acc: int,
               n_steps: int, n_substeps: int, tau: float, seed: int, n_streams: int = 0,
               use_drift: bool = False, target: int = 0, generations: float = 10.0,
               cutoff_alpha: float = 2.0) -> int:
        """Queue a VMC (mode 0) or DMC (mode 1) job; returns its id."""
        sysc, keep = pack_system(desc)
        np_ = int(desc["np"]) * int(desc["dim"])
        pos = np.ascontiguousarray(np.asarray(positions_aos, dtype=np.float64).reshape(-1, np_))
        nw = pos.shape[0]
        job = _capi.Job()
        job.system = ctypes.pointer(sysc)
        job.positions = pos.ctypes.data_as(_capi.c_dp)
        job.n_walkers = nw
        job.mode = int(mode)
        job.run = _capi.RunConfig(int(n_eq), int(n_acc), int(n_steps), int(n_substeps), float(tau),
                                  int(bool(use_drift)), int(n_streams or nw), np.uint64(seed).item(),
                                  int(target or nw), float(generations), float(cutoff_alpha))
        jid = ctypes.c_uint64()
        rc = self.lib.alea_gpu_submit_job(self.h, ctypes.byref(job), ctypes.byref(jid))
        if rc != 0:
            raise AleaGpuError(rc, self.lib.alea_gpu_server_last_error(self.h).decode())
        self._keep[jid.value] = (sysc, keep, pos, job)
        return jid.value

    def poll(self, job_id: int, timeout_ms: int = 0) -> Optional[_capi.JobResult]:
        """The job's result when it has finished, else None (after waiting
        at most timeout_ms)."""
        r = _capi.JobResult()
        rc = self.lib.alea_gpu_poll(self.h, int(job_id), int(timeout_ms), ctypes.byref(r))
        if rc == _capi.ERR_TIMEOUT:
            return None
        if rc != 0:
            raise AleaGpuError(rc, "alea_gpu_poll: unknown job")
        self._keep.pop(int(job_id), None)
        return r

    def cancel(self, job_id: int) -> bool:
        """True if the job was queued or running and is now being cancelled."""
        return self.lib.alea_gpu_cancel(self.h, int(job_id)) == 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.alea_gpu_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
