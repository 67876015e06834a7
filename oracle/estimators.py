"""Oracle restatement of the reference's observable estimators.

TEST INFRASTRUCTURE ONLY (see the package docstring).  The per-measurement
accumulation runs in liboracle.so (``o_est_gofr``, ``o_est_density``,
``o_est_sofk`` in alea_oracle.c, compiled with the reference build's FMA
contraction); the block bookkeeping and the final series restate:

* PairCorrelation  src/estimators/pair_correlation.cpp:36-220
* Density          src/estimators/density.cpp:1-281
* StructureFactor  src/estimators/structure_factor.cpp:18-225
* block_mean_error src/numerics/statistics.cpp:15-34

Each estimator keeps the per-block arrays its ``stop_block`` would store
(``history``), so tests compare them with the device's per-block output.
"""
from __future__ import annotations

import ctypes
import math
from typing import Dict, List, Sequence

import numpy as np

from .oracle import Oracle, _dp

_ip = ctypes.POINTER(ctypes.c_int)


def _lib(o: Oracle):
    lib = o.lib
    if not getattr(lib, "_est_sigs", False):
        D, L, I, P = ctypes.c_double, ctypes.c_long, ctypes.c_int, ctypes.c_void_p
        dp = ctypes.POINTER(ctypes.c_double)
        lib.o_est_gofr.argtypes = [P, dp, L, dp, D, I, dp, dp]
        lib.o_est_density.argtypes = [P, dp, L, dp, D, I, I, dp, dp]
        lib.o_est_sofk.argtypes = [P, dp, L, dp, I, _ip, _ip, dp, dp, dp, dp]
        lib._est_sigs = True
    return lib


def block_mean_error(x: Sequence[float]):
    """numerics::block_mean_error (src/numerics/statistics.cpp:15-34)."""
    m = len(x)
    if m == 0:
        return 0.0, 0.0
    s = 0.0
    for v in x:
        s += v
    mean = s / m
    if m < 2:
        return mean, 0.0
    sq = 0.0
    for v in x:
        d = v - mean
        sq += d * d
    return mean, math.sqrt(sq / (m - 1) / m)


class Gofr:
    """PairCorrelation (src/estimators/pair_correlation.cpp:36-86)."""

    def __init__(self, o: Oracle, rmax: float, n_bins: int):
        self.o, self.rmax, self.n_bins = o, float(rmax), int(n_bins)
        cell = o.setup["cell"]
        self.groups = o.setup["groups"]
        ng = len(self.groups)
        self.dim = int(o.setup["dim"])
        self.n_func = ng * (ng + 1) // 2
        self.delta = self.rmax / self.n_bins
        self.names, self.pair_count = [], []
        for a in range(ng):
            for b in range(a, ng):
                na = self.groups[a]["last"] - self.groups[a]["first"]
                nb = self.groups[b]["last"] - self.groups[b]["first"]
                self.pair_count.append(na * (na - 1) // 2 if a == b else na * nb)
                self.names.append(f"gofr_{self.groups[a]['name']}_{self.groups[b]['name']}")
        self.volume = 0.0
        if cell.get("periodic"):
            if self.rmax > cell["ws_radius"]:
                raise ValueError("gofr rmax exceeds the cell's Wigner-Seitz inradius")
            self.volume = float(cell["volume"])
        self.history: List[np.ndarray] = []
        self.start_block()

    def start_block(self):
        self.hist = np.zeros(self.n_func * self.n_bins)
        self.wsum = ctypes.c_double(0.0)

    def accumulate(self, pos_soa: np.ndarray, weights: np.ndarray):
        nw = len(weights)
        pos = np.ascontiguousarray(pos_soa, dtype=float).ravel()
        w = np.ascontiguousarray(weights, dtype=float)
        _lib(self.o).o_est_gofr(self.o.sys, _dp(pos), nw, _dp(w), self.rmax, self.n_bins,
                                _dp(self.hist), ctypes.byref(self.wsum))

    def stop_block(self):
        """pair_correlation.cpp:143-160 (no reblocking, unsigned)."""
        blk = np.zeros_like(self.hist)
        if self.wsum.value > 0.0:
            blk = self.hist * (1.0 / self.wsum.value)
        self.history.append(blk)

    def collect(self, other: "Gofr"):
        self.history.extend(other.history)

    def shell_volume(self, b: int) -> float:
        lo, hi = b * self.delta, (b + 1) * self.delta
        if self.dim == 2:
            return math.pi * (hi * hi - lo * lo)
        if self.dim == 3:
            return 4.0 / 3.0 * math.pi * (hi ** 3 - lo ** 3)
        return hi - lo

    def finalize(self) -> Dict[str, np.ndarray]:
        """pair_correlation.cpp:172-214."""
        out: Dict[str, np.ndarray] = {}
        if not self.history:
            return out
        out["gofr_r"] = (np.arange(self.n_bins) + 0.5) * self.delta
        for pid in range(self.n_func):
            pc = float(self.pair_count[pid])
            if pc == 0:
                continue
            g, ge = np.zeros(self.n_bins), np.zeros(self.n_bins)
            for b in range(self.n_bins):
                shell = self.shell_volume(b)
                norm = pc * shell / self.volume if self.volume > 0 else pc * shell
                m, e = block_mean_error([h[pid * self.n_bins + b] for h in self.history])
                g[b], ge[b] = m / norm, e / norm
            out[self.names[pid]] = g
            out[self.names[pid] + "_error"] = ge
        return out


class Density:
    """Density (src/estimators/density.cpp:13-62): block estimates streamed into
    per-cell Welford accumulators, clones merged by Chan et al."""

    def __init__(self, o: Oracle, rmax: float, n_bins: int, per_particle: bool = False):
        self.o, self.rmax, self.n_bins, self.pp = o, float(rmax), int(n_bins), bool(per_particle)
        cell = o.setup["cell"]
        self.dim = int(o.setup["dim"])
        self.periodic = bool(cell.get("periodic"))
        self.n_cells = self.n_bins ** self.dim
        self.delta = 2.0 * self.rmax / self.n_bins
        if self.periodic:
            self.cell_volume = float(cell["volume"]) / self.n_cells
        else:
            self.cell_volume = self.delta ** self.dim
        self.series = []
        for g in o.setup["groups"]:
            if self.pp:
                self.series += [f"{g['name']}_p{p - g['first']}" for p in range(g["first"], g["last"])]
            else:
                self.series.append(g["name"])
        width = len(self.series) * self.n_cells
        self.mean, self.m2, self.n_blocks = np.zeros(width), np.zeros(width), 0
        self.history: List[np.ndarray] = []
        self.start_block()

    def start_block(self):
        self.hist = np.zeros(len(self.series) * self.n_cells)
        self.wsum = ctypes.c_double(0.0)

    def accumulate(self, pos_soa: np.ndarray, weights: np.ndarray):
        nw = len(weights)
        pos = np.ascontiguousarray(pos_soa, dtype=float).ravel()
        w = np.ascontiguousarray(weights, dtype=float)
        _lib(self.o).o_est_density(self.o.sys, _dp(pos), nw, _dp(w), self.rmax, self.n_bins,
                                   int(self.pp), _dp(self.hist), ctypes.byref(self.wsum))

    def stop_block(self):
        """density.cpp:153-188 (no reblocking, unsigned)."""
        W = self.wsum.value
        norm = 1.0 / (W * self.cell_volume) if W > 0.0 else 0.0
        x = self.hist * norm
        self.history.append(x)
        self.n_blocks += 1
        if self.n_blocks == 1:
            self.mean, self.m2 = x.copy(), np.zeros_like(x)
            return
        inv_n = 1.0 / self.n_blocks
        vw = (self.n_blocks - 1) * inv_n
        d = x - self.mean
        self.mean = self.mean + d * inv_n
        self.m2 = self.m2 + d * (d * vw)

    def collect(self, other: "Density"):
        """density.cpp:190-219."""
        self.history.extend(other.history)
        if other.n_blocks == 0:
            return
        if self.n_blocks == 0:
            self.mean, self.m2, self.n_blocks = other.mean.copy(), other.m2.copy(), other.n_blocks
            return
        na, nb = float(self.n_blocks), float(other.n_blocks)
        n = na + nb
        d = other.mean - self.mean
        self.mean = self.mean + d * (nb / n)
        self.m2 = self.m2 + (other.m2 + d * (d * (na * nb / n)))
        self.n_blocks += other.n_blocks

    def finalize(self) -> Dict[str, np.ndarray]:
        """density.cpp:221-275."""
        out: Dict[str, np.ndarray] = {}
        if self.n_blocks == 0:
            return out
        n = float(self.n_blocks)
        err_norm = 1.0 / ((n - 1.0) * n) if self.n_blocks >= 2 else 0.0
        for g, name in enumerate(self.series):
            sl = slice(g * self.n_cells, (g + 1) * self.n_cells)
            out[f"density_{name}"] = self.mean[sl].copy()
            out[f"density_{name}_error"] = np.sqrt(self.m2[sl] * err_norm)
        return out


def sofk_kvectors(cell: dict, kmax: float):
    """The half-space k set of StructureFactor's constructor
    (structure_factor.cpp:18-59), sorted by |k| (stably: the reference's
    std::sort leaves the order inside a shell unspecified)."""
    b = cell["reciprocal"]
    b1, b2 = math.hypot(b[0], b[1]), math.hypot(b[2], b[3])
    nmax = int(math.ceil(kmax / min(b1, b2))) + 1
    ks = []
    for i in range(nmax + 1):
        for j in range(-nmax, nmax + 1):
            if i == 0 and j <= 0:
                continue
            kx, ky = i * b[0] + j * b[2], i * b[1] + j * b[3]
            k = math.hypot(kx, ky)
            if k <= kmax:
                ks.append((k, i, j, kx, ky))
    if not ks:
        raise ValueError("sofk: kmax is below the shortest reciprocal vector")
    ks.sort(key=lambda q: q[0])
    tol = 1e-9 * min(b1, b2)
    shell_k, shell_count, shell_of = [], [], []
    for q in ks:
        if not shell_k or q[0] - shell_k[-1] > tol:
            shell_k.append(q[0])
            shell_count.append(0)
        shell_count[-1] += 1
        shell_of.append(len(shell_k) - 1)
    return dict(n1=np.array([q[1] for q in ks], dtype=np.int32),
                n2=np.array([q[2] for q in ks], dtype=np.int32),
                kx=np.array([q[3] for q in ks]), ky=np.array([q[4] for q in ks]),
                shell_k=np.array(shell_k), shell_count=np.array(shell_count),
                shell_of=np.array(shell_of))


class Sofk:
    """StructureFactor (src/estimators/structure_factor.cpp:18-225)."""

    def __init__(self, o: Oracle, kmax: float):
        self.o = o
        cell = o.setup["cell"]
        if not cell.get("periodic") or int(o.setup["dim"]) != 2:
            raise ValueError("sofk: the structure factor needs a periodic 2-D cell")
        self.k = sofk_kvectors(cell, kmax)
        self.groups = o.setup["groups"]
        self.ng = len(self.groups)
        self.npairs = self.ng * (self.ng + 1) // 2
        self.nk = len(self.k["n1"])
        self.ns = len(self.k["shell_k"])
        self.hist_s: List[np.ndarray] = []
        self.hist_re: List[np.ndarray] = []
        self.hist_im: List[np.ndarray] = []
        self.start_block()

    def start_block(self):
        self.acc_s = np.zeros(self.npairs * self.nk)
        self.acc_re = np.zeros(self.ng * self.nk)
        self.acc_im = np.zeros(self.ng * self.nk)
        self.wsum = ctypes.c_double(0.0)

    def accumulate(self, pos_soa: np.ndarray, weights: np.ndarray):
        nw = len(weights)
        pos = np.ascontiguousarray(pos_soa, dtype=float).ravel()
        w = np.ascontiguousarray(weights, dtype=float)
        n1 = self.k["n1"].ctypes.data_as(_ip)
        n2 = self.k["n2"].ctypes.data_as(_ip)
        _lib(self.o).o_est_sofk(self.o.sys, _dp(pos), nw, _dp(w), self.nk, n1, n2, _dp(self.acc_s),
                                _dp(self.acc_re), _dp(self.acc_im), ctypes.byref(self.wsum))

    def stop_block(self):
        """structure_factor.cpp:133-163 (no reblocking, unsigned)."""
        nk, ns = self.nk, self.ns
        s = np.zeros(self.npairs * ns)
        re, im = np.zeros(self.ng * nk), np.zeros(self.ng * nk)
        W = self.wsum.value
        if W > 0.0:
            inv_w = 1.0 / W
            pid = 0
            for a in range(self.ng):
                for b in range(a, self.ng):
                    na = self.groups[a]["last"] - self.groups[a]["first"]
                    nb = self.groups[b]["last"] - self.groups[b]["first"]
                    norm = 1.0 / math.sqrt(na * nb) if na > 0 and nb > 0 else 0.0
                    for k in range(nk):
                        sh = self.k["shell_of"][k]
                        s[pid * ns + sh] += self.acc_s[pid * nk + k] * inv_w * norm / float(
                            self.k["shell_count"][sh])
                    pid += 1
            re = self.acc_re * inv_w
            im = self.acc_im * inv_w
        self.hist_s.append(s)
        self.hist_re.append(re)
        self.hist_im.append(im)

    def collect(self, other: "Sofk"):
        self.hist_s += other.hist_s
        self.hist_re += other.hist_re
        self.hist_im += other.hist_im

    def finalize(self) -> Dict[str, np.ndarray]:
        """structure_factor.cpp:176-222."""
        out: Dict[str, np.ndarray] = {}
        if not self.hist_s:
            return out

        def emit(name, hist, off, count):
            mean, err = np.zeros(count), np.zeros(count)
            for q in range(count):
                mean[q], err[q] = block_mean_error([h[off + q] for h in hist])
            out[name], out[name + "_error"] = mean, err

        out["sofk_k"] = self.k["shell_k"]
        out["sofk_shell_count"] = self.k["shell_count"].astype(float)
        pid = 0
        for a in range(self.ng):
            for b in range(a, self.ng):
                emit(f"sofk_{self.groups[a]['name']}_{self.groups[b]['name']}", self.hist_s,
                     pid * self.ns, self.ns)
                pid += 1
        out["sofk_kx"], out["sofk_ky"] = self.k["kx"], self.k["ky"]
        out["sofk_shell"] = self.k["shell_of"].astype(float)
        for g in range(self.ng):
            emit(f"rhok_{self.groups[g]['name']}_re", self.hist_re, g * self.nk, self.nk)
            emit(f"rhok_{self.groups[g]['name']}_im", self.hist_im, g * self.nk, self.nk)
        return out
