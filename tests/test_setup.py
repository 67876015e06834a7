"""Host setup (alea_setup.cpp through the C ABI) against the tables and local
energies of the compiled reference's builders.

The breakup coefficients need not agree bit for bit (the optimized fit
amplifies rounding differences of the quadrature to ~1e-8 relative, the
reference's own breakup tolerance), but the physics they encode must: the
local energy of every fixture walker agrees with the reference-built system
to 1e-10 relative, through the oracle, on the CPU.
"""
import json
import os

import numpy as np
import pytest

from conftest import golden

alea_setup = pytest.importorskip("alea_b200.setup")

CASES = {
    "heg42": ("heg2d", dict(n_up=21, n_down=21, rs=30.0, pade_b=0.3)),
    "heg10": ("heg2d", dict(n_up=5, n_down=5, rs=30.0, pade_b=0.3)),
    "crystal16": ("crystal2d", dict(nx=4, ny=4, rs=40.0, gauss_c=0.1)),
    "dipoles16": ("dipoles2d", dict(n=16, rs=0.03526184897173477)),
}

E_L_RTOL = 1e-10        # local energy, reference-built vs this setup
TABLE_RTOL = 1e-7       # breakup tables (fit conditioning), relative to max|.|
INIT_SEED = 12345       # the seed the eval fixtures' walkers were drawn with


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    fn, kw = CASES[request.param]
    s = getattr(alea_setup, fn)(**kw)
    return request.param, s, golden(f"setup_{request.param}.json")


def _close(a, b, rtol):
    a, b = np.asarray(a, float), np.asarray(b, float)
    assert a.shape == b.shape
    scale = max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)
    assert np.max(np.abs(a - b)) <= rtol * scale if a.size else True


def test_cell_orbitals_cusps(case):
    name, s, g = case
    d = s.desc
    _close(d["cell"]["vectors"], g["cell"]["vectors"], 1e-15)
    assert [(x["first"], x["last"], x["charge"]) for x in d["groups"]] == \
        [(x["first"], x["last"], x["charge"]) for x in g["groups"]]
    for mb, gb in zip(d.get("slater", []), g.get("slater", [])):
        assert mb["type"] == gb["type"]
        if gb["type"] == "plane_wave":
            _close(mb["k"], gb["k"], 1e-15)
            assert mb["is_sin"] == gb["is_sin"]
        else:
            _close(mb["centers"], gb["centers"], 1e-15)
            _close(mb["alphas"], gb["alphas"], 1e-15)
    for mp, gp in zip(d.get("pade", []), g.get("pade", [])):
        assert (mp["ga"], mp["gb"]) == (gp["ga"], gp["gb"])
        _close(mp["a"], gp["a"], 1e-15)
        _close(mp["b"], gp["b"], 1e-15)
    for mz, gz in zip(d.get("zero_energy", []), g.get("zero_energy", [])):
        for k in ("ga", "gb", "b", "exponent", "matching_radius"):
            assert mz[k] == gz[k]
        assert mz["cutoff"] == pytest.approx(gz["cutoff"], rel=1e-15)
    for mi, gi in zip(d.get("inverse_power", []), g.get("inverse_power", [])):
        assert (mi["ga"], mi["gb"], mi["strength"], mi["exponent"]) == \
            (gi["ga"], gi["gb"], gi["strength"], gi["exponent"])
        assert mi["tail"] == pytest.approx(gi["tail"], rel=1e-12)
    assert len(d.get("zero_energy", [])) == len(g.get("zero_energy", []))
    assert len(d.get("inverse_power", [])) == len(g.get("inverse_power", []))
    for md, gd in zip(d.get("drummond", []), g.get("drummond", [])):
        assert md["pairs"] == gd["pairs"] and md["C"] == gd["C"]
        assert md["gamma"] == pytest.approx(gd["gamma"], rel=1e-15)
        assert md["L"] == pytest.approx(gd["L"], rel=1e-15)


def test_breakup_tables(case):
    name, s, g = case
    d = s.desc
    if "ewald" not in g:
        assert "ewald" not in d
        return
    pairs = [(d["ewald"], g["ewald"])]
    pairs += [(a["image_sum"], b["image_sum"]) for a, b in zip(d.get("pade", []), g.get("pade", []))
              if "image_sum" in b]
    for mine, ref in pairs:
        assert mine["n1"] == ref["n1"] and mine["n2"] == ref["n2"]
        _close(mine["kx"], ref["kx"], 1e-15)
        _close(mine["weight"], ref["weight"], TABLE_RTOL)
        sp, rp = mine["spline"], ref["spline"]
        assert sp["n_knots"] == rp["n_knots"]
        _close(sp["scaled"], rp["scaled"], TABLE_RTOL)
    if "self_energy" in g["ewald"]:
        assert d["ewald"]["self_energy"] == pytest.approx(g["ewald"]["self_energy"], rel=TABLE_RTOL)


def test_parameter_breakup_tables(case):
    """The optimisable Padé parameter (b) of each image-summed term: its
    index, du/db's limit and the breakup of du/db - limit on the same k set
    (PadeJastrow::build_image_sum, pade_jastrow.cpp:214-248)."""
    name, s, ref = case
    for mine, theirs in zip(s.desc.get("pade", []), ref.get("pade", [])):
        assert len(mine.get("opt", [])) == len(theirs.get("opt", []))
        for o, r in zip(mine.get("opt", []), theirs.get("opt", [])):
            assert int(o["index"]) == int(r["index"])
            assert abs(o["inf"] - r["inf"]) <= 1e-12 * abs(r["inf"])
            _close(o["weight"], r["weight"], TABLE_RTOL)
            _close(o["spline"]["scaled"], r["spline"]["scaled"], TABLE_RTOL)


def test_local_energy_matches_reference_tables(case):
    from oracle import Oracle
    name, s, g = case
    ev = golden(f"eval_{name}.json")
    pos = np.array(ev["positions"])
    el = []
    for desc in (s.desc, g):
        o = Oracle(desc)
        o.init(pos, capacity=len(pos))
        el.append(np.array([o.measure(i) for i in range(len(pos))]))
    np.testing.assert_allclose(el[0], el[1], rtol=E_L_RTOL)
    np.testing.assert_allclose(el[1], ev["local_energy"], rtol=E_L_RTOL)


def test_initial_positions(case):
    name, s, g = case
    ev = golden(f"eval_{name}.json")
    pos = np.array(ev["positions"])
    mine = s.positions(INIT_SEED, len(pos)).reshape(pos.shape)
    np.testing.assert_allclose(mine, pos, rtol=0, atol=1e-12 * np.max(np.abs(pos)))


def test_exciton_setup():
    s = alea_setup.exciton2d()
    g = golden("setup_exciton.json")
    assert s.desc["pade"][0]["a"] == g["pade"][0]["a"]
    assert s.desc["coulomb"][0]["coef"] == g["coulomb"][0]["coef"]
    ev = golden("eval_exciton.json")
    ref = np.array(ev["positions"])
    pos = s.positions(INIT_SEED, len(ref)).reshape(ref.shape)
    np.testing.assert_array_equal(pos, ref)


def test_setup_rejects_bad_input():
    with pytest.raises(ValueError):
        alea_setup.heg2d(0, 0, 30.0)
    with pytest.raises(ValueError, match="shell"):
        alea_setup.heg2d(4, 4, 30.0)        # 4 plane waves leave a shell open
    with pytest.raises(ValueError):
        alea_setup.crystal2d(4, 3, 30.0)    # odd row count


MADELUNG_2D_SQUARE = 1.6155426267   # tests/test_ewald.cpp:212-225 of the reference


def _madelung_system(tol=1e-8):
    # ±1 charges on a square lattice of spacing 1: (0,0)+ (1,1)+ | (1,0)- (0,1)- in a 2x2 cell
    s = alea_setup.charges2d([2.0, 0.0, 0.0, 2.0], [2, 2], [1.0, -1.0], ewald_tol=tol)
    pos = np.array([[0.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0, 1.0]])
    return s, pos


def test_ewald_reproduces_square_madelung_constant():
    """E = -(N/2) M q²/a for N = 4 ions: the reference's Madelung known answer,
    through this library's breakup tables and the oracle's Ewald sum."""
    from oracle import Oracle
    s, pos = _madelung_system()
    o = Oracle(s.desc)
    o.init(pos)
    M = -2.0 * o.measure(0) / 4.0
    assert M == pytest.approx(MADELUNG_2D_SQUARE, abs=1e-6)
    # periodic translation of one ion by a lattice vector leaves E unchanged
    moved = pos.copy()
    moved[0, 2] += 3 * 2.0
    moved[0, 3] -= 2 * 2.0
    o.init(moved)
    assert -2.0 * o.measure(0) / 4.0 == pytest.approx(M, abs=1e-12)


def test_with_backflow_builds_the_reference_apps_backflow_gas():
    """with_backflow on the 5 + 5 gas gives the reference App's backflow
    description of that system (channels, truncation, zero slope, cutoff at
    the inradius, free parameters) as recorded in the heg10bf fixture."""
    import json
    from alea_b200 import setup as S
    from conftest import golden
    d = S.with_backflow(S.heg2d(5, 5, 30.0).desc)
    assert json.dumps(d["backflow"]) == json.dumps(golden("setup_heg10bf.json")["backflow"])
    assert "slater" not in d
