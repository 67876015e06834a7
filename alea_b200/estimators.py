"""Host side of the device estimators: the reference's finalize().

The device accumulates every measurement and the C ABI returns one block
estimate per block and chain (``alea_gpu_estimator_blocks``, the arrays the
reference's ``stop_block`` stores).  These functions turn them into the named
series of the reference's ``RunResult``:

* g(r)     PairCorrelation::finalize  (src/estimators/pair_correlation.cpp:172-214)
* density  Density::stop_block/collect/finalize (src/estimators/density.cpp:153-275):
           per-cell Welford over a chain's blocks, chains merged in order by
           Chan et al.'s rule, as VMC reduces its thread clones
           (src/qmc/vmc.cpp:381-387)
* S(k)     StructureFactor::finalize (src/estimators/structure_factor.cpp:176-222)

Errors are the block standard errors of numerics::block_mean_error
(src/numerics/statistics.cpp:15-34), blocks of all chains in chain order.
"""
from __future__ import annotations

import math
from typing import Any, Dict, List, Sequence

import numpy as np

KINDS = {"gofr": 1, "density": 2, "sofk": 3}


def block_mean_error(x: np.ndarray):
    """Mean and standard error of the mean of per-block values along axis 0."""
    x = np.asarray(x, dtype=float)
    m = x.shape[0]
    mean = x.sum(axis=0) / m
    if m < 2:
        return mean, np.zeros_like(mean)
    sq = ((x - mean) ** 2).sum(axis=0)
    return mean, np.sqrt(sq / (m - 1) / m)


def _pairs(groups: Sequence[Dict[str, Any]]):
    for a in range(len(groups)):
        for b in range(a, len(groups)):
            yield a, b


def finalize_gofr(blocks: np.ndarray, groups, rmax: float, n_bins: int, volume: float,
                  dim: int = 2) -> Dict[str, np.ndarray]:
    """blocks [n_blocks_total][n_pairs * n_bins], chain-major."""
    out: Dict[str, np.ndarray] = {}
    if len(blocks) == 0:
        return out
    delta = rmax / n_bins
    out["gofr_r"] = (np.arange(n_bins) + 0.5) * delta
    lo = np.arange(n_bins) * delta
    hi = (np.arange(n_bins) + 1) * delta
    shell = math.pi * (hi * hi - lo * lo) if dim == 2 else 4.0 / 3.0 * math.pi * (hi ** 3 - lo ** 3)
    for pid, (a, b) in enumerate(_pairs(groups)):
        na = groups[a]["last"] - groups[a]["first"]
        nb = groups[b]["last"] - groups[b]["first"]
        pc = na * (na - 1) // 2 if a == b else na * nb
        if pc == 0:
            continue
        norm = pc * shell / volume if volume > 0 else pc * shell
        m, e = block_mean_error(blocks[:, pid * n_bins:(pid + 1) * n_bins])
        name = f"gofr_{groups[a]['name']}_{groups[b]['name']}"
        out[name] = m / norm
        out[name + "_error"] = e / norm
    return out


def density_series_names(groups, per_particle: bool) -> List[str]:
    names = []
    for g in groups:
        if per_particle:
            names += [f"{g['name']}_p{p - g['first']}" for p in range(g["first"], g["last"])]
        else:
            names.append(g["name"])
    return names


def finalize_density(chain_blocks: np.ndarray, groups, n_bins: int, per_particle: bool = False
                     ) -> Dict[str, np.ndarray]:
    """chain_blocks [n_chains][n_blocks][n_series * n_cells]."""
    out: Dict[str, np.ndarray] = {}
    mean = m2 = None
    n_total = 0
    for chain in chain_blocks:
        # Welford over this chain's blocks (density.cpp:153-188)
        cm, c2, n = None, None, 0
        for x in chain:
            n += 1
            if n == 1:
                cm, c2 = x.copy(), np.zeros_like(x)
                continue
            inv_n = 1.0 / n
            d = x - cm
            cm = cm + d * inv_n
            c2 = c2 + d * (d * ((n - 1) * inv_n))
        if n == 0:
            continue
        if n_total == 0:
            mean, m2, n_total = cm, c2, n
            continue
        # Chan merge (density.cpp:190-219)
        na, nb = float(n_total), float(n)
        tot = na + nb
        d = cm - mean
        mean = mean + d * (nb / tot)
        m2 = m2 + (c2 + d * (d * (na * nb / tot)))
        n_total += n
    if n_total == 0:
        return out
    n_cells = n_bins * n_bins
    err_norm = 1.0 / ((n_total - 1.0) * n_total) if n_total >= 2 else 0.0
    for s, name in enumerate(density_series_names(groups, per_particle)):
        sl = slice(s * n_cells, (s + 1) * n_cells)
        out[f"density_{name}"] = mean[sl].copy()
        out[f"density_{name}_error"] = np.sqrt(m2[sl] * err_norm)
    return out


def finalize_sofk(blocks: np.ndarray, groups, kvec: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """blocks [n_blocks_total][n_pairs * n_shells + 2 * n_groups * n_k], chain-major."""
    out: Dict[str, np.ndarray] = {}
    if len(blocks) == 0:
        return out
    ns, nk, ng = len(kvec["shell_k"]), len(kvec["n1"]), len(groups)
    npairs = ng * (ng + 1) // 2
    out["sofk_k"] = kvec["shell_k"]
    out["sofk_shell_count"] = kvec["shell_count"].astype(float)
    for pid, (a, b) in enumerate(_pairs(groups)):
        m, e = block_mean_error(blocks[:, pid * ns:(pid + 1) * ns])
        name = f"sofk_{groups[a]['name']}_{groups[b]['name']}"
        out[name], out[name + "_error"] = m, e
    out["sofk_kx"], out["sofk_ky"] = kvec["kx"], kvec["ky"]
    out["sofk_shell"] = kvec["shell_of"].astype(float)
    base = npairs * ns
    for g in range(ng):
        for part, off in (("re", base + g * nk), ("im", base + (ng + g) * nk)):
            m, e = block_mean_error(blocks[:, off:off + nk])
            name = f"rhok_{groups[g]['name']}_{part}"
            out[name], out[name + "_error"] = m, e
    return out


NAMESPACES = ("gofr", "density", "sofk", "rhok")


def relabel(series: Dict[str, np.ndarray], label: str) -> Dict[str, np.ndarray]:
    """Insert an output label after each key's namespace, as the reference's
    Estimator::write_results does (src/estimators/estimator.h:110-131):
    label "fw0" turns gofr_up_down into gofr_fw0_up_down."""
    out = {}
    for k, v in series.items():
        ns = max((n for n in NAMESPACES if k == n or k.startswith(n + "_")), key=len, default=None)
        out[k if ns is None else ns + "_" + label + k[len(ns):]] = v
    return out
