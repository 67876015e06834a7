"""Host setup of the systems the walker kernels run, through the C ABI.

Each builder returns a :class:`Setup`: ``desc`` is the system description dict
that :func:`alea_b200.pack_system` and :class:`alea_b200.Walkers` take, and
``positions(seed, nw)`` draws initial walkers as the reference App does
(src/qmc/app.cpp:56-112).  The tables (plane-wave shells, Ewald and
image-summed Padé breakups, cusps) are computed by ``alea_setup.cpp`` inside
``libalea_b200.so``.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import _capi


class Setup:
    def __init__(self, handle: ctypes.c_void_p):
        self._lib = _capi.load()
        self._h = handle
        self.desc = json.loads(self._lib.alea_gpu_setup_json(handle).decode())

    def positions(self, seed: int, nw: int) -> np.ndarray:
        """Initial walkers, AoS [nw, np, dim]."""
        np_, dim = int(self.desc["np"]), int(self.desc["dim"])
        out = np.zeros((nw, np_, dim), dtype=np.float64)
        rc = self._lib.alea_gpu_setup_positions(self._h, ctypes.c_uint64(seed), nw,
                                                out.ctypes.data_as(_capi.c_dp))
        if rc != 0:
            raise ValueError(f"alea_gpu_setup_positions failed ({rc})")
        return out

    def close(self):
        if self._h:
            self._lib.alea_gpu_setup_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _make(fn, *args) -> Setup:
    lib = _capi.load()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(512)
    rc = getattr(lib, fn)(*args, ctypes.byref(h), err, len(err))
    if rc != 0:
        raise ValueError(f"{fn}: {err.value.decode()}")
    return Setup(h)


def heg2d(n_up: int, n_down: int, rs: float, pade_b: float = 0.3, pade_a: float = 0.0,
          ewald_tol: float = 1e-6) -> Setup:
    """2-D electron gas (square cell, plane waves, image-summed Padé, Ewald)."""
    return _make("alea_gpu_setup_heg2d", n_up, n_down, rs, pade_b, pade_a, ewald_tol)


def heg2d_twisted(n_up: int, n_down: int, rs: float, twist, pade_b: float = 0.3, pade_a: float = 0.0,
                  ewald_tol: float = 1e-6) -> Setup:
    """2-D electron gas at a twist (t_x, t_y) in units of the reciprocal
    vectors: twisted plane waves, complex determinant (real at an integer twist)."""
    return _make("alea_gpu_setup_heg2d_twisted", n_up, n_down, rs, pade_b, pade_a, float(twist[0]),
                 float(twist[1]), ewald_tol)


def crystal2d(nx: int, ny: int, rs: float, gauss_c: float = 0.1, alpha0: float = 0.0,
              cutoff_frac: float = 0.999, jitter: float = 0.0, ewald_tol: float = 1e-6) -> Setup:
    """2-D Wigner crystal (triangular sites, Gaussians, Drummond, Ewald)."""
    return _make("alea_gpu_setup_crystal2d", nx, ny, rs, gauss_c, alpha0, cutoff_frac, jitter,
                 ewald_tol)


def charges2d(lattice, counts, charges, ewald_tol: float = 1e-6) -> Setup:
    """Point charges in a periodic 2-D cell, Ewald Coulomb only."""
    lat = np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).ravel())
    cnt = np.ascontiguousarray(np.asarray(counts, dtype=np.int32))
    q = np.ascontiguousarray(np.asarray(charges, dtype=np.float64))
    if lat.size != 4 or cnt.size != q.size:
        raise ValueError("charges2d: lattice needs 4 numbers, one charge per group")
    return _make("alea_gpu_setup_charges2d", lat.ctypes.data_as(_capi.c_dp), int(cnt.size),
                 cnt.ctypes.data_as(_capi.c_ip), q.ctypes.data_as(_capi.c_dp), ewald_tol)


def ewald3d(lattice, ewald_tol: float = 1e-6) -> Setup:
    """The 3-D Coulomb Ewald tables of a periodic cell (rows of `lattice`, 3x3):
    host tables only, in `desc["ewald"]` (the walker kernels are 2-D)."""
    lat = np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).ravel())
    if lat.size != 9:
        raise ValueError("ewald3d: lattice needs 9 numbers")
    return _make("alea_gpu_setup_ewald3d", lat.ctypes.data_as(_capi.c_dp), ewald_tol)


def heg3d(n_up: int, n_down: int, rs: float, bf_like: float = 0.1, bf_unlike: float = 0.1,
          bf_cut: float = 0.0, alpha0: float = 0.0, ewald_tol: float = 1e-6) -> Setup:
    """3-D electron gas with backflow determinants, Drummond Jastrows and the
    3-D Ewald sum (alea_gpu_setup_heg3d)."""
    return _make("alea_gpu_setup_heg3d", n_up, n_down, rs, bf_like, bf_unlike, bf_cut, alpha0, ewald_tol)


def dipoles2d(n: int, rs: float, strength: float = 1.0, exponent: float = 3.0,
              matching_radius: float = 0.0459) -> Setup:
    """2-D dipolar bosons: zero-energy Jastrow, C/r^p with its continuum tail."""
    return _make("alea_gpu_setup_dipoles2d", n, rs, strength, exponent, matching_radius)


def exciton2d(L_init: float = 1.0) -> Setup:
    """Open 2-D exciton with the exact trial function (E = -1)."""
    lib = _capi.load()
    h = ctypes.c_void_p()
    rc = lib.alea_gpu_setup_exciton2d(L_init, ctypes.byref(h))
    if rc != 0:
        raise ValueError(f"alea_gpu_setup_exciton2d failed ({rc})")
    return Setup(h)


def with_backflow(desc: dict, c0_like: float = 0.3, c0_unlike: float = 0.2, c1_unlike: float = 0.002,
                  C: int = 3, cutoff: float = 0.0) -> dict:
    """A copy of a plane-wave system description whose determinants become
    backflow determinants (BackflowSlaterDeterminant with the
    transformation of backflow_transformation.h): each block is displaced by
    every block, through η(r) = (1 - r/L)^C (c_0 + c_1 r), like-spin channels
    with zero slope at the origin (c_1 = C c_0/L, only c_0 free) and
    unlike-spin channels with c_0 and c_1 free.  The cutoff defaults to the
    cell's Wigner-Seitz inradius, the largest the reference allows."""
    import copy
    out = copy.deepcopy(desc)
    blocks = out.pop("slater")
    if any(b.get("type") != "plane_wave" for b in blocks):
        raise ValueError("with_backflow: plane-wave determinants only")
    v = np.asarray(out["cell"]["vectors"], float).reshape(2, 2)
    L = cutoff or 0.5 * min(np.linalg.norm(v[0]), np.linalg.norm(v[1]), np.linalg.norm(v[0] + v[1]),
                            np.linalg.norm(v[0] - v[1]))
    out["backflow"] = []
    for b in blocks:
        chans = []
        for src in blocks:
            like = src["first"] == b["first"]
            chans.append({"source_first": src["first"], "source_last": src["last"], "C": C,
                          "coeffs": [c0_like, C * c0_like / L] if like else [c0_unlike, c1_unlike],
                          "L": L, "zero_slope": 1 if like else 0, "opt_index": [0] if like else [0, 1]})
        out["backflow"].append({"first": b["first"], "last": b["last"], "type": "plane_wave", "k": b["k"],
                                "is_sin": b["is_sin"], "channels": chans})
    return out
