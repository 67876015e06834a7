"""d ln psi / d p of the pair Jastrows' optimisable parameters (the linear
method's O_k), through the C ABI, against the compiled reference's
compute_parameter_derivatives on the same walkers (eval fixtures: the
reference's App walkers, seed 12345).

The electron gases' image-summed Padé terms each carry one optimisable
parameter (b; a_1 is fixed by the cusp): the short-range sum of du/db minus
its breakup, plus the k-space part from each walker's rho(k).  The crystal
variant frees its Drummond alpha_0, an alpha_2 term and the cutoff L, and
each Gaussian block's shared width (d ln det/d alpha = Tr(A dD), and
dA = -A dD A for the curvature term).  The backflow gas frees each channel's
c_0 (and the unlike-spin c_1): O = Σ_P Σ_j (F_P · r_Pj) dη(r_Pj)/dp with the
committed F = A^T ∇φ(x); its curvature terms follow the quasi-coordinates'
parameter tangent through A, F, T, G and the Jacobian columns (a channel of
truncation C < 3 is refused, as the reference reports none).  Tolerance 1e-10
relative to the largest |O_k|; after VMC steps (rho(k) updated move by move)
the derivatives equal those of a fresh evaluation of the same positions.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

SYSTEMS = ["heg10", "heg42", "heg10t", "heg10bf", "crystal16p"]


def ours(setup, components):
    """The reference's components whose parameters this library computes, in
    its order: the backflow determinants with free channel parameters, or the
    determinant when a Gaussian block's width is free, then the pair terms
    (Padé per spin pair, or the crystal's Drummond items)."""
    n_terms = len(setup.get("pade", [])) + len(setup.get("drummond", []))
    bf = setup.get("backflow", [])
    det = [components[d] for d, b in enumerate(bf) if any(ch.get("opt_index") for ch in b["channels"])]
    if any(b.get("opt_alpha") for b in setup.get("slater", [])):
        det = [components[0]]
    return det + components[-n_terms:]


@pytest.mark.parametrize("name", SYSTEMS)
def test_parameter_derivatives_match_reference(name):
    import alea_b200
    setup = golden(f"setup_{name}.json")
    ev = golden(f"eval_{name}.json")
    pos = np.array(ev["positions"])
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(pos)
    got = g.parameter_derivatives()
    want = np.concatenate([np.array(d).reshape(-1, len(pos)) for d in ours(setup, ev["param_derivs"])])
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-10 * np.abs(want).max()


def test_parameter_derivatives_follow_the_walk():
    import alea_b200
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"])
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(pos)
    g.set_streams(9, alea_b200.STREAM_VMC, 4)
    for _ in range(3):
        g.vmc_step(225.0, 2)
    moved = g.parameter_derivatives()
    f = alea_b200.Walkers(setup, capacity=8)
    f.upload(g.download()["positions"].reshape(len(pos), -1, 2))
    fresh = f.parameter_derivatives()
    assert np.max(np.abs(moved - fresh)) <= 1e-10 * np.abs(fresh).max()


@pytest.mark.parametrize("name", SYSTEMS)
def test_parameter_gradient_derivatives_match_reference(name):
    """d(grad ln psi)/dp and d(lap ln psi)/dp (the linear method's curvature
    term) against compute_parameter_gradient_derivatives, 1e-9 relative."""
    import alea_b200
    setup = golden(f"setup_{name}.json")
    ev = golden(f"eval_{name}.json")
    pos = np.array(ev["positions"])
    nw, m = len(pos), int(setup["np"]) * int(setup["dim"])
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(pos)
    dg, dl = g.parameter_gradient_derivatives()
    terms = ours(setup, ev["param_grad_derivs"])
    assert all(t["ok"] for t in terms)
    wg = np.concatenate([np.array(t["grad"]).reshape(-1, m, nw) for t in terms])
    wl = np.concatenate([np.array(t["lap"]).reshape(-1, m, nw) for t in terms])
    assert dg.shape == wg.shape and dl.shape == wl.shape
    assert np.max(np.abs(dg - wg)) <= 1e-9 * np.abs(wg).max()
    assert np.max(np.abs(dl - wl)) <= 1e-9 * np.abs(wl).max()


def test_backflow_curvature_refused_below_truncation_three():
    """A channel with C = 2 (η'' jumps at L): no curvature term, as in the
    reference (supports_parameter_gradient_derivatives is false there)."""
    import copy
    import alea_b200
    setup = copy.deepcopy(golden("setup_heg10bf.json"))
    for b in setup["backflow"]:
        for ch in b["channels"]:
            ch["C"] = 2
            if ch.get("zero_slope"):
                ch["coeffs"][1] = 2.0 * ch["coeffs"][0] / ch["L"]
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(np.array(golden("eval_heg10bf.json")["positions"]))
    with pytest.raises(alea_b200.AleaGpuError) as e:
        g.parameter_gradient_derivatives()
    assert e.value.code == 3
    g.close()


def test_backflow_curvature_matches_finite_differences_at_42():
    """The benchmark gas (21 + 21 electrons, r_s = 30) with backflow
    determinants: each free channel parameter's d(grad ln psi)/dp and
    d(lap ln psi)/dp against central differences of the evaluated
    derivatives at p +- h (h = 1e-5 |p|; the Jastrow does not depend on p),
    1e-6 relative to the largest entry."""
    import copy
    import alea_b200
    from alea_b200 import setup as S
    base = S.heg2d(21, 21, 30.0)
    desc = S.with_backflow(base.desc)
    pos = base.positions(31, 4)
    g = alea_b200.Walkers(desc, capacity=4)
    g.upload(pos)
    dg, dl = g.parameter_gradient_derivatives()
    g.close()
    q = 0
    for d, blk in enumerate(desc["backflow"]):
        for c, ch in enumerate(blk["channels"]):
            for slot in ch["opt_index"]:
                h = 1e-5 * abs(ch["coeffs"][slot])
                side = []
                for sgn in (1.0, -1.0):
                    e = copy.deepcopy(desc)
                    cc = e["backflow"][d]["channels"][c]
                    cc["coeffs"][slot] += sgn * h            # c_0 (zero slope: c_1 follows) or c_1
                    if cc["zero_slope"]:
                        cc["coeffs"][1] = cc["C"] * cc["coeffs"][0] / cc["L"]
                    w = alea_b200.Walkers(e, capacity=4)
                    w.upload(pos)
                    o = w.download()
                    side.append((o["grad"].T, o["lap"].T))
                    w.close()
                fg = (side[0][0] - side[1][0]) / (2 * h)
                fl = (side[0][1] - side[1][1]) / (2 * h)
                assert np.max(np.abs(dg[q] - fg)) <= 1e-6 * np.abs(fg).max(), (d, c, slot)
                assert np.max(np.abs(dl[q] - fl)) <= 1e-6 * np.abs(fl).max(), (d, c, slot)
                q += 1
    assert q == 6
