"""The 3-D Coulomb Ewald tables (alea_gpu_setup_ewald3d, this project's own
breakup with the 3-D radial kernel; the reference refuses 3-D Ewald) against
the known answers of cubic crystals: the Madelung constants of rock salt
(NaCl, 1.747564594633) and caesium chloride (CsCl, 1.762674773070), from
E = Σ_{i<j} q_i q_j [1/r − f_l(r)] (minimum image, r < r_c) + Σ_k w_k |ρ(k)|²
− ½ f_l(0) Σ q_i², evaluated from the tables alone (oracle/ewald3d.py), to 5e-8 (the
breakup's 20 knots leave ~1e-8; the reference's 2-D known answer is held to
1e-6).
"""
import numpy as np
import pytest

from alea_b200 import setup as S
from oracle import ewald3d


def _energy(lattice, pos, q, e):
    return ewald3d.energy(lattice, pos, q, e)


@pytest.fixture(scope="module")
def cubic():
    s = S.ewald3d(np.eye(3), ewald_tol=1e-10)
    yield s.desc
    s.close()


def test_rock_salt_madelung_constant(cubic):
    na = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]], float)
    cl = na + np.array([.5, 0, 0])
    pos = np.concatenate([na, cl])
    q = np.array([1.0] * 4 + [-1.0] * 4)
    E = _energy(np.eye(3), pos, q, cubic["ewald"])
    # E = -(N pairs) M / d with 4 ion pairs and the nearest distance d = 1/2
    assert -E * 0.5 / 4.0 == pytest.approx(1.747564594633, abs=5e-8)


def test_caesium_chloride_madelung_constant(cubic):
    pos = np.array([[0, 0, 0], [.5, .5, .5]], float)
    q = np.array([1.0, -1.0])
    E = _energy(np.eye(3), pos, q, cubic["ewald"])
    d = np.sqrt(3.0) / 2.0
    assert -E * d == pytest.approx(1.762674773070, abs=5e-8)


def test_translation_and_neutral_background(cubic):
    """A rigid shift of every ion leaves E unchanged; a uniform background
    enters only through Σq (zero here)."""
    pos = np.array([[0, 0, 0], [.5, .5, .5]], float)
    q = np.array([1.0, -1.0])
    e0 = _energy(np.eye(3), pos, q, cubic["ewald"])
    e1 = _energy(np.eye(3), pos + np.array([0.137, -0.29, 0.41]), q, cubic["ewald"])
    assert e1 == pytest.approx(e0, rel=1e-10)
