"""Oracle of the 3-D Ewald sum: the electrostatic energy of point charges in a
periodic 3-D cell from the breakup tables alone.

TEST INFRASTRUCTURE ONLY (see the package docstring).  The reference refuses
3-D Ewald (src/numerics/ewald_breakup.cpp:211-213); its 2-D sum
(src/hamiltonian/ewald_term.cpp:368-612) has the same three parts, restated
here for three dimensions:

    E = Σ_{i<j} q_i q_j [1/r − f_l(r)]   (minimum image, r < r_c)
      + Σ_k w_k |ρ(k)|²                   (half-space k, ρ(k) = Σ_i q_i e^{ik·r_i})
      − ½ f_l(0) Σ q_i²  − ½ (Σ q_i)² f̃_s(0)/V

with f_l the breakup's quintic-Hermite long-range spline.  Pinned by the
rock-salt and caesium-chloride Madelung constants (tests/test_ewald3d.py).
"""
from __future__ import annotations

import numpy as np


def _hermite(t):
    u = 1.0 - t
    return np.array([u ** 3 * (1 + 3 * t + 6 * t * t), t * u ** 3 * (1 + 3 * t), 0.5 * t * t * u ** 3])


def f_long(sp, r: float) -> float:
    """The breakup's quintic Hermite long-range part at r < r_c (value,
    δ·f', δ²·f'' per knot, mirrored basis on the right knot)."""
    s = np.array(sp["scaled"]).reshape(-1, 3)
    x = r * sp["inv_delta"]
    i = min(int(x), sp["n_knots"] - 2)
    t = x - i
    hl, hr = _hermite(t), _hermite(1.0 - t)
    return float(s[i] @ hl + s[i + 1] @ (hr * np.array([1.0, -1.0, 1.0])))


def energy(lattice, pos, q, e) -> float:
    """E of charges q at positions pos [n][3] in the cell of lattice rows
    (9 numbers), with the tables e of alea_gpu_setup_ewald3d / _heg3d."""
    lat = np.asarray(lattice, float).reshape(3, 3)
    inv = np.linalg.inv(lat)
    pos = np.asarray(pos, float).reshape(-1, 3)
    q = np.asarray(q, float)
    rc = e["r_cut"]
    er = 0.0
    for i in range(len(q)):
        for j in range(i + 1, len(q)):
            d = pos[i] - pos[j]
            f = d @ inv
            d = (f - np.rint(f)) @ lat
            r = float(np.linalg.norm(d))
            if r < rc:
                er += q[i] * q[j] * (1.0 / r - f_long(e["spline"], r))
    k = np.stack([e["kx"], e["ky"], e["kz"]], axis=1)
    rho = np.exp(1j * pos @ k.T).T @ q
    ek = float(np.sum(np.array(e["weight"]) * np.abs(rho) ** 2))
    self_ = -0.5 * e["v_long_zero"] * float(np.sum(q * q))
    bg = -0.5 * float(np.sum(q)) ** 2 * e["sr_k0"]
    return er + ek + self_ + bg
