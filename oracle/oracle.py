"""ctypes wrapper for the oracle restatement and runner for the compiled reference.

Test infrastructure only (see the package docstring).
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from typing import Any, Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB: Optional[ctypes.CDLL] = None

# scalar slots of an oracle walker record (alea_oracle.c, enum S_*)
S_LOGPSI, S_EL, S_WEIGHT, S_EPREV, S_RRP, S_RRA, S_AGE, S_ID, S_PARENT, S_ERR, S_ELI = range(11)


def load_oracle_lib() -> ctypes.CDLL:
    """Load (building if needed) liboracle.so."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(HERE, "liboracle.so")
    src = os.path.join(HERE, "alea_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "oracle", "REF_CC=gcc"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(path)
    P, D, L, I, U = (ctypes.c_void_p, ctypes.c_double, ctypes.c_long, ctypes.c_int,
                     ctypes.c_uint64)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.o_sys_new.restype = P
    lib.o_sys_new.argtypes = [dp, L]
    lib.o_sys_free.argtypes = [P]
    lib.o_layout.argtypes = [P, ctypes.POINTER(ctypes.c_long)]
    lib.o_init.argtypes = [P, dp, L, dp]
    lib.o_measure.argtypes = [P, dp]
    lib.o_move.argtypes = [P, dp, I, dp, I, dp]
    lib.o_vmc.argtypes = [P, dp, L, I, U, I, I, I, I, D, I, dp, dp]
    lib.o_dmc.argtypes = [P, dp, ctypes.POINTER(ctypes.c_long), L, I, U, I, I, I, I, D, D, L,
                          dp, dp, L]
    lib.o_splitmix64.restype = U
    lib.o_splitmix64.argtypes = [U]
    lib.o_stream_seed.restype = U
    lib.o_stream_seed.argtypes = [U, U, U]
    lib.o_xoshiro_raw.argtypes = [ctypes.POINTER(ctypes.c_uint64), L,
                                  ctypes.POINTER(ctypes.c_uint64)]
    lib.o_rng_draws.argtypes = [U, L, I, dp]
    lib.o_ziggurat_tables.argtypes = [ctypes.POINTER(ctypes.c_uint64), dp, dp, dp]
    _LIB = lib
    return lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def blob_from_setup(sd: Dict[str, Any]) -> np.ndarray:
    """Flatten a system description (the ref_harness ``setup`` JSON schema,
    also produced by the product's host setup) into the oracle's blob
    (layout documented at blob_read() in alea_oracle.c)."""
    out: List[float] = []
    dim = int(sd["dim"])
    cell = sd["cell"]
    out += [dim, int(sd["np"]), int(cell["periodic"])]
    if cell["periodic"]:
        out += list(cell["vectors"])
    out.append(len(sd["groups"]))
    for g in sd["groups"]:
        out += [g["first"], g["last"], g["charge"]] + list(g["inv_mass"])
    blocks = sd.get("slater", [])
    out.append(len(blocks))
    for b in blocks:
        btype = {"plane_wave": 0, "gaussian": 1, "twisted_plane_wave": 2}[b["type"]]
        out += [b["first"], b["last"], btype]
        if b["type"] == "plane_wave":
            out += list(b["k"]) + list(b["is_sin"])
        elif b["type"] == "twisted_plane_wave":
            out += list(b["q"])
        else:
            out += list(b["centers"]) + list(b["alphas"])
    terms = []
    for p in sd.get("pade", []):
        t = [0, 1, p["ga"][0], p["ga"][1], p["gb"][0], p["gb"][1], len(p["a"]), len(p["b"])]
        t += list(p["a"]) + list(p["b"])
        im = p.get("image_sum")
        if im:
            sp = im["spline"]
            t += [1, sp["r_cut"], sp["inv_delta"], sp["n_knots"]] + list(sp["scaled"])
            t += [im["u_inf"], len(im["weight"])]
            t += list(im["n1"]) + list(im["n2"]) + list(im["kx"]) + list(im["ky"]) + list(im["weight"])
        else:
            t += [0]
        terms.append(t)
    for d in sd.get("drummond", []):
        t = [1, len(d["pairs"])]
        for pr in d["pairs"]:
            t += list(pr)
        t += [d["C"], d["gamma"], d["L"], len(d["coeffs"])] + list(d["coeffs"])
        terms.append(t)
    for z in sd.get("zero_energy", []):
        t = [2, 1, z["ga"][0], z["ga"][1], z["gb"][0], z["gb"][1], z["b"], z["exponent"],
             z["matching_radius"], z["cutoff"]]
        t += list(bessel_k01_chebyshev())
        terms.append(t)
    out.append(len(terms))
    for t in terms:
        out += t
    ew = sd.get("ewald")
    if ew:
        sp = ew["spline"]
        out += [1, sp["r_cut"], sp["inv_delta"], sp["n_knots"]] + list(sp["scaled"])
        out += [ew["r_cut"], ew["inv_eps"], ew["self_energy"] + ew["background_energy"],
                len(ew["weight"])]
        out += list(ew["n1"]) + list(ew["n2"]) + list(ew["weight"])
    else:
        out.append(0)
    cl = sd.get("coulomb", [])
    out.append(len(cl))
    for c in cl:
        out += [c["ga"][0], c["ga"][1], c["gb"][0], c["gb"][1], c["coef"]]
    ip = sd.get("inverse_power", [])
    out.append(len(ip))
    for c in ip:
        out += [c["ga"][0], c["ga"][1], c["gb"][0], c["gb"][1], c["strength"], c["exponent"], c["tail"]]
    bf = sd.get("backflow", [])
    out.append(len(bf))
    for b in bf:
        out += [b["first"], b["last"], 0 if b["type"] == "plane_wave" else 1]
        if b["type"] == "plane_wave":
            out += list(b["k"]) + list(b["is_sin"])
        else:
            out += list(b["centers"]) + list(b["alphas"])
        out.append(len(b["channels"]))
        for c in b["channels"]:
            out += [c["source_first"], c["source_last"], c["C"], c["L"], len(c["coeffs"])] + list(c["coeffs"])
    return np.asarray(out, dtype=np.float64)


def bessel_k01_chebyshev(terms: int = 24) -> np.ndarray:
    """Chebyshev coefficients of sqrt(x) e^x K_nu(x), nu = 0, 1, in xi = 4/x - 1
    (numerics/scaled_bessel_k01.h: projection on 8 x terms first-kind nodes),
    from scipy's k0e/k1e.  Order 0 in [0, terms), order 1 in [terms, 2 terms)."""
    from scipy.special import k0e, k1e
    m = 8 * terms
    theta = np.pi * (np.arange(m) + 0.5) / m
    x = 4.0 / (np.cos(theta) + 1.0)
    f0 = np.sqrt(x) * k0e(x)
    f1 = np.sqrt(x) * k1e(x)
    c = np.zeros(2 * terms)
    for k in range(terms):
        ck = np.cos(k * theta)
        norm = (1.0 if k == 0 else 2.0) / m
        c[k] = norm * np.sum(f0 * ck)
        c[terms + k] = norm * np.sum(f1 * ck)
    return c


class Oracle:
    """One system in the oracle restatement, with a block of walker records."""

    def __init__(self, setup: Dict[str, Any]):
        self.lib = load_oracle_lib()
        self.setup = setup
        self._blob = blob_from_setup(setup)
        self.sys = self.lib.o_sys_new(_dp(self._blob), len(self._blob))
        if not self.sys:
            raise ValueError("oracle: malformed system description")
        lay = (ctypes.c_long * 12)()
        self.lib.o_layout(self.sys, lay)
        (self.W, self.o_pos, self.o_dist, self.o_grad, self.o_lap, self.o_scal,
         self.o_lpc, self.o_gc, self.o_lc, self.ncomp, self.o_pgrad, self.o_plap) = list(lay)
        self.np = int(setup["np"])
        self.dim = int(setup["dim"])
        self.walkers = np.zeros((0, self.W))

    def __del__(self):
        try:
            self.lib.o_sys_free(self.sys)
        except Exception:
            pass

    # walker record views
    def pos(self, i=None):
        n = self.np * self.dim
        v = self.walkers[:, self.o_pos:self.o_pos + n]
        return v if i is None else v[i]

    def grad(self):
        n = self.np * self.dim
        return self.walkers[:, self.o_grad:self.o_grad + n]

    def phase_grad(self):
        n = self.np * self.dim
        return self.walkers[:, self.o_pgrad:self.o_pgrad + n] if self.o_pgrad >= 0 else None

    def phase_lap(self):
        n = self.np * self.dim
        return self.walkers[:, self.o_plap:self.o_plap + n] if self.o_plap >= 0 else None

    def lap(self):
        n = self.np * self.dim
        return self.walkers[:, self.o_lap:self.o_lap + n]

    def scalar(self, k):
        return self.walkers[:, self.o_scal + k]

    def init(self, pos_aos: np.ndarray, capacity: Optional[int] = None) -> None:
        pos_aos = np.ascontiguousarray(pos_aos, dtype=np.float64).reshape(len(pos_aos), -1)
        nw = pos_aos.shape[0]
        cap = max(capacity or nw, nw)
        self.walkers = np.zeros((cap, self.W))
        self.lib.o_init(self.sys, _dp(self.walkers), nw, _dp(pos_aos))
        self.nw = nw

    def move(self, iw: int, p: int, new_pos, accept: bool) -> np.ndarray:
        out = np.zeros(2 + 2 * self.dim)
        rec = self.walkers[iw]
        npos = np.asarray(new_pos, dtype=np.float64)
        self.lib.o_move(self.sys, _dp(rec), p, _dp(npos), 1 if accept else 0, _dp(out))
        return out

    def measure(self, iw: int) -> float:
        self.lib.o_measure(self.sys, _dp(self.walkers[iw]))
        return float(self.walkers[iw, self.o_scal + S_EL])

    def vmc(self, threads, seed, n_eq, n_acc, n_steps, n_substeps, tau, drift=False):
        nw = self.nw
        steps = (n_eq + n_acc) * n_steps
        el = np.zeros(steps * nw)
        stats = np.zeros(2)
        self.lib.o_vmc(self.sys, _dp(self.walkers), nw, threads, seed, n_eq, n_acc, n_steps,
                       n_substeps, tau, 1 if drift else 0, _dp(el), _dp(stats))
        return el.reshape(steps, nw), stats

    def dmc(self, threads, seed, n_eq, n_acc, n_steps, n_substeps, tau, target,
            generations=10.0):
        nw = ctypes.c_long(self.nw)
        steps = (n_eq + n_acc) * n_steps
        trace = np.zeros(steps * 5)
        cap = self.walkers.shape[0]
        rc = self.lib.o_dmc(self.sys, _dp(self.walkers), ctypes.byref(nw), cap, threads, seed,
                            n_eq, n_acc, n_steps, n_substeps, tau, generations, target,
                            _dp(trace), None, 0)
        if rc != 0:
            raise RuntimeError("oracle dmc: capacity too small")
        self.nw = nw.value
        return trace.reshape(steps, 5)


def ref_harness_path() -> Optional[str]:
    p = os.path.join(HERE, "_ref", "ref_harness")
    return p if os.path.exists(p) else None


def run_ref_harness(mode: str, **kw) -> Dict[str, Any]:
    exe = ref_harness_path()
    if exe is None:
        raise FileNotFoundError("oracle/_ref/ref_harness is not built")
    args = [exe, mode] + [f"{k}={v}" for k, v in kw.items()]
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    res = subprocess.run(args, check=True, capture_output=True, text=True, env=env)
    return json.loads(res.stdout)
