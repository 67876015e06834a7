"""Walker-population checkpoints: the reference's walkers_out / walkers_in.

The reference serialises a population to HDF5 (io::write_walkers /
read_walkers, src/io/walker_io.h:34-65): one flat dataset "positions" of
nw·np·dim doubles in AoS row order [w][p][d], attributes n_walkers,
n_particles, dim, the cell's lattice_vectors (absent for an open cell) and,
for milestone snapshots, tag and blocks_done.  HDF5 is not available to this
package, so the same fields are written to a NumPy .npz archive; a host that
has the reference's HDF5 layer writes the rows of
``Walkers.final_configurations()`` with io::write_walkers instead.

Loading applies the reference's walkers_in checks (src/qmc/app.cpp:834-866):
a particle-count or dimension mismatch is fatal, and so is a cell that
differs from the run's by more than 1e-9 (1 + |a|) in any lattice entry.
"""
from __future__ import annotations

import os
from typing import Any, Dict, Optional, Sequence

import numpy as np


class CheckpointError(RuntimeError):
    pass


def write_walkers(path: str, rows: np.ndarray, lattice: Optional[Sequence[float]] = None,
                  tag: str = "", blocks_done: int = -1) -> None:
    """rows [nw][np][dim] (Walkers.final_configurations()).  Written to a
    temporary name and renamed, so a crash never leaves a torn file."""
    rows = np.asarray(rows, dtype=np.float64)
    if rows.ndim != 3:
        raise ValueError("rows must be [walkers][particles][dim]")
    nw, npart, dim = rows.shape
    fields: Dict[str, Any] = dict(positions=rows.ravel(), n_walkers=nw, n_particles=npart, dim=dim,
                                  lattice_vectors=np.asarray(lattice if lattice is not None else [],
                                                             dtype=np.float64))
    if tag:
        fields["tag"] = np.array(tag)
    if blocks_done >= 0:
        fields["blocks_done"] = blocks_done
    tmp = path + ".tmp.npz"
    np.savez(tmp, **fields)
    os.replace(tmp, path)


def read_walkers(path: str) -> Dict[str, Any]:
    """The stored population; CheckpointError on a missing or malformed file
    (a continuation must never fall back to random positions)."""
    try:
        with np.load(path, allow_pickle=False) as z:
            nw, npart, dim = int(z["n_walkers"]), int(z["n_particles"]), int(z["dim"])
            pos = np.array(z["positions"], dtype=np.float64)
            lat = np.array(z["lattice_vectors"], dtype=np.float64)
            out = dict(nw=nw, np=npart, dim=dim, lattice=lat,
                       tag=str(z["tag"]) if "tag" in z else "",
                       blocks_done=int(z["blocks_done"]) if "blocks_done" in z else -1)
    except (OSError, KeyError, ValueError) as exc:
        raise CheckpointError(f"walkers checkpoint {path!r}: {exc}") from exc
    if nw < 1 or pos.size != nw * npart * dim:
        raise CheckpointError(f"walkers checkpoint {path!r}: positions do not hold {nw} x {npart} x {dim}")
    out["positions"] = pos.reshape(nw, npart, dim)
    return out


def check_compatible(wf: Dict[str, Any], desc: Dict[str, Any]) -> None:
    """The walkers_in checks of src/qmc/app.cpp:834-866 against a system
    description (the dict of alea_b200.setup / the golden setups)."""
    npart, dim = int(desc["np"]), int(desc["dim"])
    if wf["np"] != npart or wf["dim"] != dim:
        raise CheckpointError(f"walkers_in: geometry mismatch: file has np={wf['np']} dim={wf['dim']}, "
                              f"run needs np={npart} dim={dim}")
    cell = desc["cell"]
    cellv = np.asarray(cell["vectors"], dtype=np.float64) if cell.get("periodic") else np.zeros(0)
    lat = np.asarray(wf["lattice"], dtype=np.float64)
    if lat.size != cellv.size or np.any(np.abs(lat - cellv) > 1e-9 * (1.0 + np.abs(cellv))):
        raise CheckpointError("walkers_in: simulation-cell mismatch between the checkpoint and this run")
