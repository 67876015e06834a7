"""The device path on the benchmark's own systems, against the compiled
reference's drivers (fixtures from tests/golden/make_fixtures.py).

* heg42: the N = 42, r_s = 30 electron gas of the DMC benchmark, through the
  one-warp sweep: DMC::run with one crowd per walker (populations and block
  energies), and DMC/VMC with fewer streams than walkers (the crowd split:
  each stream walks a contiguous range), bit for bit where the reference's
  decisions are bitwise (VMC positions, branching counts).
* crystal120: the 10 x 12 Wigner crystal (60 + 60 electrons, Gaussian
  orbitals, Drummond Jastrow, Ewald) on the generic sweep: evaluation and VMC
  steps against the reference, and a DMC step of 8192 walkers.
* the heg42 DMC energy against a long reference DMC run, within 2 sigma.

Tolerances: local energies and block energies 1e-10 relative; positions after
drift moves 1e-9 relative; populations exact.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b, floor=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def ref_blocks(r):
    p = r["params"]
    n_eq = p["eq"] * p["steps"]
    ws = np.array(r["weight_sum"])
    we = np.array(r["weighted_energy_sum"])
    return [we[b * p["steps"]:(b + 1) * p["steps"]].sum() / ws[b * p["steps"]:(b + 1) * p["steps"]].sum()
            for b in range(p["acc"])], n_eq


def walkers(desc, capacity):
    import alea_b200
    return alea_b200.Walkers(desc, capacity=capacity)


@pytest.mark.parametrize("fixture", ["dmc_heg42", "dmc_heg42_crowd"])
def test_heg42_dmc_matches_reference(fixture):
    """DMC::run on the benchmark system: block energies to 1e-10 (every
    step's weighted sums, so the same branching history), the same final
    population and its configurations to 1e-9."""
    r = golden(f"{fixture}.json")
    p = r["params"]
    nw = p["nw"]
    threads = p.get("threads", nw)
    setup = golden("setup_heg42.json")
    g = walkers(setup, 2 * nw + 2)
    g.upload(np.array(r["initial_positions"]))
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], threads, p["seed"],
                            target=nw)
    want, _ = ref_blocks(r)
    assert rel(blocks, want) < 1e-10
    fin = np.array(r["final_positions"]).reshape(-1, 42 * 2)
    assert g.nw == fin.shape[0]
    d = g.download()
    assert np.max(np.abs(d["positions"] - fin)) < 1e-9 * np.abs(fin).max()
    g.close()


def test_heg42_vmc_crowds_match_reference():
    """VMC::run with 4 threads over 64 walkers (16 per stream): accept
    decisions and so positions bit for bit, every thread's block energies."""
    r = golden("vmc_heg42_crowd.json")
    p = r["params"]
    g = walkers(golden("setup_heg42.json"), p["nw"])
    g.upload(np.array(r["initial_positions"]))
    res, blocks = g.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["threads"], p["seed"])
    fin = np.array(r["final_positions"]).reshape(p["nw"], -1)
    assert np.array_equal(g.download()["positions"], fin)
    assert res.acceptance == pytest.approx(r["acceptance"], rel=1e-15)
    assert rel(blocks, r["block_energies"]) < 1e-10
    assert res.energy == pytest.approx(r["energy"], rel=1e-10)
    g.close()


def test_crystal120_evaluate_and_vmc_match_reference():
    """The 120-electron crystal (generic CTA sweep, 60 x 60 determinants):
    ln|psi| differences and E_L of the reference App's walkers, then two VMC
    steps with one stream per walker."""
    import alea_b200
    setup = golden("setup_crystal120.json")
    ev = golden("eval_crystal120.json")
    pos = np.array(ev["positions"])
    g = walkers(setup, len(pos))
    g.upload(pos)
    d = g.download()
    assert rel(d["local_energy"], ev["local_energy"]) < 1e-10
    lp, lr = d["log_psi"], np.array(ev["log_psi"])
    assert np.max(np.abs((lp - lp[0]) - (lr - lr[0]))) < 1e-9 * max(1.0, np.abs(lr).max())
    g.close()
    r = golden("vmc_crystal120.json")
    p = r["params"]
    g = walkers(setup, p["nw"])
    g.upload(np.array(r["initial_positions"]))
    res, blocks = g.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["nw"], p["seed"])
    fin = np.array(r["final_positions"]).reshape(p["nw"], -1)
    assert np.array_equal(g.download()["positions"], fin)
    assert res.acceptance == pytest.approx(r["acceptance"], rel=1e-15)
    assert rel(blocks, r["block_energies"]) < 1e-10
    g.close()


def test_crystal120_dmc_step_at_8192_walkers():
    """The crystal benchmark's population: 8192 walkers from the lattice
    sites with N(0, 0.1 r_s) jitter, a VMC step, then a DMC advance and
    branch; every energy finite and the population within the clip window."""
    import alea_b200
    from alea_b200 import setup as S
    nw = 8192
    s = S.crystal2d(10, 12, 40.0, gauss_c=0.1, jitter=0.1 * 40.0)
    pos = s.positions(2024, nw)
    g = walkers(s.desc, 2 * nw + 2)
    g.upload(pos)
    g.set_streams(3, alea_b200.STREAM_VMC, nw)
    g.vmc_step(400.0, 1, False)
    el = g.download()["local_energy"]
    assert np.all(np.isfinite(el))
    e0 = float(np.mean(el))
    g.set_streams(4, alea_b200.STREAM_DMC, nw)
    st = g.dmc_advance(1.0, 1, e0, e0, 10.0, 15.0)
    assert st.n_walkers == nw and np.isfinite(st.energy_sum) and st.n_accepted > 0
    g.dmc_branch(np.array([1, 2, 3, 4], dtype=np.uint64), nw)
    assert nw // 5 + 1 <= g.nw <= 2 * nw + 1
    assert np.all(np.isfinite(g.download()["local_energy"]))
    g.close()
    s.close()


def test_heg42_dmc_energy_agrees_with_reference_statistically():
    """The benchmark system's DMC energy: a device run from an independent
    start and seed against the compiled reference's DMC::run (1024 walkers,
    8 crowds, tau 0.5): block means within 2 combined standard errors."""
    from alea_b200 import setup as S
    ref = golden("dmcstat_heg42.json")
    p = ref["params"]
    g = walkers(golden("setup_heg42.json"), 2 * p["nw"] + 2)
    g.upload(S.heg2d(21, 21, 30.0).positions(4242, p["nw"]))
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["threads"],
                            seed=4243, target=p["nw"], generations=10.0)
    assert len(blocks) == p["acc"] and np.all(np.isfinite(blocks))
    sigma = float(np.hypot(res.energy_error, ref["energy_error"]))
    assert res.energy_error > 0 and abs(res.energy - ref["energy"]) < 2.0 * sigma, \
        (res.energy, res.energy_error, ref["energy"], ref["energy_error"])
    g.close()


def test_heg42_vmc_energy_agrees_with_reference_statistically():
    """The VMC benchmark's shape (512 walkers, 8 streams, Metropolis step
    0.5 r_s, 5 sweeps per step): the device's VMC energy from an independent
    start and seed against the compiled reference's VMC::run, within 2
    combined standard errors."""
    from alea_b200 import setup as S
    ref = golden("vmcstat_heg42.json")
    p = ref["params"]
    g = walkers(golden("setup_heg42.json"), p["nw"])
    g.upload(S.heg2d(21, 21, 30.0).positions(5151, p["nw"]))
    res, blocks = g.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["threads"], 5152)
    sigma = float(np.hypot(res.energy_error, ref["energy_error"]))
    assert res.energy_error > 0 and abs(res.energy - ref["energy"]) < 2.0 * sigma, \
        (res.energy, res.energy_error, ref["energy"], ref["energy_error"])
    assert abs(res.acceptance - ref["acceptance"]) < 0.02
    g.close()
