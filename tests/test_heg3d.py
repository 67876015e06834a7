"""Three-dimensional walkers (alea_bf3d.cu): the backflow electron gas of the
benchmark's fourth configuration (54 electrons, r_s = 5) and smaller gases,
and the open 3-D cell of the reference's own 3-D backflow test (Gaussian
orbitals, two backflow channels, a Padé Jastrow, open Coulomb), against the
compiled reference's own dimension-generic components and drivers
(BackflowSlaterDeterminant, DrummondJastrow, PadeJastrow, Kinetic,
CoulombTerm, VMC::run, DMC::run,
fixtures from tests/golden/make_fixtures.py; the reference builds no 3-D
plane-wave shells and has no 3-D Ewald, so its systems carry the plane waves
directly and the kinetic energy alone).  The 3-D Ewald energy is checked
against the oracle's restatement (oracle/ewald3d.py, pinned by Madelung
constants).

Known answer: a determinant of plane waves without Jastrow or backflow has
E_L = Σ_k k²/2 exactly.

The DMC runs use cusp-free Jastrows (Drummond with Γ = 0): with the
kinetic energy alone, a Coulomb cusp leaves an unbalanced 1/r local energy
whose weights overflow within a step.

Tolerances: ln|psi| differences, gradients, Laplacians and E_L 1e-10
relative (1e-9 for Laplacians); Metropolis VMC positions bit for bit;
drift-move positions 1e-9; DMC block energies 1e-10 and identical
populations.
"""
import numpy as np
import pytest

from conftest import golden


def rel(a, b, floor=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


# ─────────────────────────── CPU: fixtures and host setup ──────────────────


def test_plane_wave_kinetic_known_answer_in_reference_fixture():
    """The reference's own E_L of the plain 54-electron plane-wave
    determinant (no Jastrow, no backflow) is Σ k²/2 for every walker."""
    s = golden("setup_heg54pw3d.json")
    ev = golden("eval_heg54pw3d.json")
    k2 = sum(float(np.sum(np.array(b["k"]) ** 2)) for b in s["slater"])
    assert np.allclose(ev["local_energy"], 0.5 * k2, rtol=1e-12, atol=0)
    assert np.allclose(ev["kinetic"], 0.5 * k2, rtol=1e-12, atol=0)


def test_open_gaussian_fixture_potential():
    """The open 3-D fixture's E_L minus its kinetic part is the open Coulomb
    attraction between the three particles and the two holes."""
    ev = golden("eval_gauss3d.json")
    for w, pos in enumerate(ev["positions"]):
        x = np.array(pos).reshape(5, 3)
        v = sum(-1.0 / np.linalg.norm(x[i] - x[j]) for i in range(3) for j in range(3, 5))
        assert ev["local_energy"][w] - ev["kinetic"][w] == pytest.approx(v, rel=1e-12)


def test_host_setup_matches_reference_system():
    """alea_gpu_setup_heg3d builds the fixture's system: the same cubic cell,
    plane waves (shell order, cos/sin), backflow channels and Drummond terms;
    its 3-D Ewald tables meet the Madelung-pinned energy formula."""
    from alea_b200 import setup as S
    ref = golden("setup_heg54bf3d.json")
    st = S.heg3d(27, 27, 5.0, bf_like=0.1, bf_unlike=0.1, alpha0=-0.01)
    d = st.desc
    assert np.allclose(d["cell"]["vectors"], ref["cell"]["vectors"], rtol=1e-15)
    for a, b in zip(d["backflow"], ref["backflow"]):
        assert (a["first"], a["last"]) == (b["first"], b["last"])
        assert np.allclose(a["k"], b["k"], rtol=0, atol=1e-15)
        assert list(map(int, a["is_sin"])) == list(map(int, b["is_sin"]))
        for ca, cb in zip(a["channels"], b["channels"]):
            assert (ca["source_first"], ca["source_last"], ca["C"]) == (cb["source_first"], cb["source_last"], cb["C"])
            assert np.allclose(ca["coeffs"], cb["coeffs"], rtol=1e-15)
            assert ca["L"] == pytest.approx(cb["L"], rel=1e-15)
    for a, b in zip(d["drummond"], ref["drummond"]):
        assert (a["C"], a["gamma"]) == (b["C"], b["gamma"])
        assert a["L"] == pytest.approx(b["L"], rel=1e-15)
        assert [list(map(int, p)) for p in a["pairs"]] == [list(map(int, p)) for p in b["pairs"]]
    # the constant of the sum: self and background energies of 54 unit charges
    e = d["ewald"]
    assert e["self_energy"] == pytest.approx(-0.5 * e["v_long_zero"] * 54, rel=1e-15)
    assert e["background_energy"] == pytest.approx(-0.5 * 54 ** 2 * e["sr_k0"], rel=1e-15)
    pos = st.positions(7, 3)
    assert pos.shape == (3, 54, 3)
    L = d["cell"]["vectors"][0]
    assert np.all(np.abs(pos) <= 0.5 * L)
    st.close()


# ─────────────────────────── GPU: against the reference ────────────────────


def walkers(desc, capacity):
    import alea_b200
    return alea_b200.Walkers(desc, capacity=capacity)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["heg54bf3d", "heg14bf3d", "heg54pw3d", "gauss3d"])
def test_evaluate_matches_reference(name):
    setup = golden(f"setup_{name}.json")
    ev = golden(f"eval_{name}.json")
    pos = np.array(ev["positions"])
    g = walkers(setup, len(pos))
    g.upload(pos)
    d = g.download()
    nw, n = len(pos), setup["np"] * 3
    assert rel(d["local_energy"], ev["local_energy"]) < 1e-10
    lp, lr = d["log_psi"], np.array(ev["log_psi"])
    assert np.max(np.abs((lp - lp[0]) - (lr - lr[0]))) < 1e-10 * max(1.0, np.abs(lr).max())
    gr = np.array(ev["grad"]).reshape(n, nw).T
    assert np.max(np.abs(d["grad"] - gr)) < 1e-10 * max(1.0, np.abs(gr).max())
    lr_ = np.array(ev["lap"]).reshape(n, nw).T
    assert np.max(np.abs(d["lap"] - lr_)) < 1e-9 * max(1.0, np.abs(lr_).max())
    if name == "heg54pw3d":
        k2 = sum(float(np.sum(np.array(b["k"]) ** 2)) for b in setup["slater"])
        assert np.allclose(d["local_energy"], 0.5 * k2, rtol=1e-12, atol=0)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["heg54bf3d", "heg14bf3d", "heg14bf3d_drift", "heg54pw3d", "gauss3d",
                                  "gauss3d_drift"])
def test_vmc_matches_reference(name):
    r = golden(f"vmc_{name}.json")
    p = r["params"]
    g = walkers(golden(f"setup_{r['system']}.json"), p["nw"])
    g.upload(np.array(r["initial_positions"]))
    res, blocks = g.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["nw"], p["seed"],
                            drift=bool(p.get("drift", 0)))
    fin = np.array(r["final_positions"]).reshape(p["nw"], -1)
    got = g.download()["positions"]
    if p.get("drift", 0):
        assert np.max(np.abs(got - fin)) < 1e-9 * np.abs(fin).max()
    else:
        assert np.array_equal(got, fin)
    assert res.acceptance == pytest.approx(r["acceptance"], rel=1e-15)
    assert rel(blocks, r["block_energies"]) < 1e-10
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["heg14bf3ds", "heg54bf3ds", "gauss3d"])
def test_dmc_matches_reference(name):
    r = golden(f"dmc_{name}.json")
    p = r["params"]
    nw = p["nw"]
    g = walkers(golden(f"setup_{name}.json"), 4 * nw + 4)
    g.upload(np.array(r["initial_positions"]))
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"], target=nw)
    ws = np.array(r["weight_sum"])            # the accumulation steps' sums
    we = np.array(r["weighted_energy_sum"])
    want = [we[b * p["steps"]:(b + 1) * p["steps"]].sum() / ws[b * p["steps"]:(b + 1) * p["steps"]].sum()
            for b in range(p["acc"])]
    assert rel(blocks, want) < 1e-10
    fin = np.array(r["final_positions"]).reshape(-1, golden(f"setup_{name}.json")["np"] * 3)
    assert g.nw == fin.shape[0]
    assert np.max(np.abs(g.download()["positions"] - fin)) < 1e-9 * np.abs(fin).max()
    g.close()


@pytest.mark.gpu
def test_ewald_potential_matches_oracle():
    """The benchmark system with its 3-D Ewald sum: E_L minus the same
    walkers' E_L without it is the oracle's electrostatic energy."""
    from alea_b200 import setup as S
    from oracle import ewald3d
    st = S.heg3d(27, 27, 5.0)
    d = st.desc
    pos = st.positions(11, 4)
    full = walkers(d, 4)
    full.upload(pos)
    e_full = full.download()["local_energy"]
    bare = dict(d)
    bare.pop("ewald")
    kin = walkers(bare, 4)
    kin.upload(pos)
    e_kin = kin.download()["local_energy"]
    q = np.full(54, -1.0)
    want = [ewald3d.energy(d["cell"]["vectors"], pos[w].reshape(54, 3), q, d["ewald"]) for w in range(4)]
    assert rel(e_full - e_kin, want) < 1e-10
    full.close()
    kin.close()
    st.close()


@pytest.mark.gpu
def test_benchmark_population_dmc_step():
    """The fourth configuration's shape: 4096 walkers of the 54-electron
    backflow gas with 3-D Ewald, a VMC step and a DMC advance + branch; every
    energy finite, the population within the clip window."""
    import alea_b200
    from alea_b200 import setup as S
    nw = 4096
    st = S.heg3d(27, 27, 5.0)
    g = walkers(st.desc, 2 * nw + 2)
    g.upload(st.positions(2025, nw))
    g.set_streams(3, alea_b200.STREAM_VMC, nw)
    g.vmc_step(1.0, 1, False)
    e = g.download()["local_energy"]
    assert np.all(np.isfinite(e))
    g.set_streams(5, alea_b200.STREAM_DMC, nw)
    et = float(np.mean(e))
    st_ = g.dmc_advance(0.02, 1, et, et, 1e30, 1e30)
    assert np.isfinite(st_.energy_sum)
    g.dmc_branch(np.array([1, 2, 3, 4], dtype=np.uint64), nw)
    assert nw // 5 + 1 <= g.nw <= 2 * nw + 1
    g.close()
    st.close()


# ─────────────────────────── GPU: what 3-D contexts refuse, rows in 3-D ─────

UNSUPPORTED = 3   # ALEA_ERR_UNSUPPORTED


def _small3d():
    return golden("setup_heg14bf3d.json"), np.array(golden("eval_heg14bf3d.json")["positions"])


@pytest.mark.gpu
def test_refused_three_dimensional_systems():
    """A 3-D cell must be orthorhombic along the axes, a 3-D determinant has
    at most 32 rows, and 3-D Padé terms are minimum-image only."""
    import copy
    import alea_b200
    setup, _ = _small3d()
    skew = copy.deepcopy(setup)
    v = list(skew["cell"]["vectors"])
    v[1] = 0.5 * v[0]
    skew["cell"]["vectors"] = v
    with pytest.raises(alea_b200.AleaGpuError, match="orthorhombic") as e:
        walkers(skew, 4)
    assert e.value.code == UNSUPPORTED
    pw = golden("setup_heg54pw3d.json")
    big = copy.deepcopy(pw)
    b = big["slater"][0]
    b["last"] = b["first"] + 33
    b["k"] = list(b["k"]) + [0.0] * (6 * 3)
    b["is_sin"] = list(b["is_sin"]) + [0] * 6
    big["slater"][1]["first"] = 33
    big["np"] = 33 + 27
    big["groups"][0]["last"] = 33
    big["groups"][1]["first"], big["groups"][1]["last"] = 33, 60
    big["slater"][1]["last"] = 60
    with pytest.raises(alea_b200.AleaGpuError, match="1..32 rows") as e:
        walkers(big, 4)
    assert e.value.code == UNSUPPORTED
    pade = copy.deepcopy(golden("setup_gauss3d.json"))
    pade["pade"][0]["image_sum"] = {"spline": {"r_cut": 1.0, "inv_delta": 1.0, "n_knots": 2, "scaled": [0.0] * 6},
                                    "u_inf": 0.0, "n1": [1], "n2": [0], "kx": [1.0], "ky": [0.0], "weight": [0.0]}
    with pytest.raises(alea_b200.AleaGpuError) as e:
        walkers(pade, 4)
    assert e.value.code in (1, UNSUPPORTED)   # an image sum in an open cell is invalid either way


@pytest.mark.gpu
def test_two_dimensional_entry_points_refuse_3d_contexts():
    """Single moves, the FP32 form, the allocation-free step, estimators,
    forward walking and parameter derivatives answer ALEA_ERR_UNSUPPORTED for
    a 3-D context, which then still steps."""
    import alea_b200
    setup, pos = _small3d()
    g = walkers(setup, len(pos))
    g.upload(pos)
    g.set_streams(5, alea_b200.STREAM_VMC, len(pos))
    calls = [lambda: g.move(0, pos.reshape(len(pos), -1, 3)[:, 0, :]),
             lambda: g.set_precision("fp32"),
             lambda: g.vmc_step_noalloc(1.0, 1, False),
             lambda: g.add_estimator("gofr", n_bins=8, rmax=1.0),
             lambda: g.set_forward_walking([1.0]),
             lambda: g.parameter_derivatives()]
    for call in calls:
        with pytest.raises(alea_b200.AleaGpuError) as e:
            call()
        assert e.value.code == UNSUPPORTED
    st = g.vmc_step(1.0, 1, False)
    assert st.n_walkers == len(pos) and np.all(np.isfinite(g.download()["local_energy"]))
    g.close()


@pytest.mark.gpu
def test_configuration_rows_round_trip_in_3d():
    """final_configurations gives AoS rows [w][p][3]; seeding a second
    context with them reproduces the positions and local energies."""
    setup, pos = _small3d()
    a = walkers(setup, len(pos))
    a.upload(pos)
    rows = a.final_configurations()
    assert rows.shape == (len(pos), setup["np"], 3)
    np.testing.assert_array_equal(rows.reshape(len(pos), -1), a.download()["positions"])
    b = walkers(setup, len(pos))
    b.seed_walker_rows(rows, len(pos))
    da, db = a.download(), b.download()
    np.testing.assert_array_equal(db["positions"], da["positions"])
    np.testing.assert_array_equal(db["local_energy"], da["local_energy"])
    a.close()
    b.close()


@pytest.mark.gpu
def test_served_3d_job_equals_its_own_run():
    """A 3-D VMC job through the serving queue (per-job contexts, footprint
    admission) gives its own alea_gpu_vmc_run result bit for bit beside a
    2-D job."""
    import alea_b200
    setup, pos = _small3d()
    nw = len(pos)
    g = walkers(setup, nw)
    g.upload(pos)
    own, _ = g.vmc_run(1, 2, 3, 1, 1.0, nw, 77)
    g.close()
    srv = alea_b200.Server(max_running=2)
    two = golden("setup_heg10.json")
    other = srv.submit(two, np.array(golden("eval_heg10.json")["positions"]), 0, 1, 2, 3, 1, 225.0, seed=5)
    jid = srv.submit(setup, pos, 0, 1, 2, 3, 1, 1.0, seed=77)
    r = srv.poll(jid, timeout_ms=120000)
    assert r is not None and r.status == 0
    assert r.result.energy == own.energy and r.result.energy_error == own.energy_error
    assert r.result.acceptance == own.acceptance and r.result.n_moves == own.n_moves
    assert r.footprint_bytes > 0
    assert srv.poll(other, timeout_ms=120000).status == 0
    srv.close()
    # a packing server runs it on a context of its own (the packed sweeps are two-dimensional)
    srv = alea_b200.Server(max_running=2, packed=True)
    jid = srv.submit(setup, pos, 0, 1, 2, 3, 1, 1.0, seed=77)
    r = srv.poll(jid, timeout_ms=120000)
    assert r is not None and r.status == 0
    assert r.result.energy == own.energy and r.result.n_moves == own.n_moves
    srv.close()


@pytest.mark.gpu
def test_dmc_energy_agrees_with_reference_statistically():
    """The 14-electron 3-D gas with its backflow determinant alone (kinetic
    energy only): the device's DMC energy from an independent start and seed
    against a long DMC::run of the compiled reference (1024 walkers, 40
    blocks of 10 steps, tau = 0.5), within 2 combined standard errors."""
    from alea_b200 import setup as S
    ref = golden("dmcstat_heg14bf3dp.json")
    p = ref["params"]
    st = S.heg3d(7, 7, 5.0)
    start = st.positions(4244, p["nw"])
    st.close()
    g = walkers(golden("setup_heg14bf3dp.json"), 2 * p["nw"] + 2)
    g.upload(start)
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["threads"],
                            seed=4245, target=p["nw"], generations=10.0)
    assert len(blocks) == p["acc"] and np.all(np.isfinite(blocks))
    sigma = float(np.hypot(res.energy_error, ref["energy_error"]))
    assert res.energy_error > 0 and abs(res.energy - ref["energy"]) < 2.0 * sigma, \
        (res.energy, res.energy_error, ref["energy"], ref["energy_error"])
    g.close()
