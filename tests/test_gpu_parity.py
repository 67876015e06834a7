"""GPU path vs the oracle, through the C ABI (libalea_b200.so).

Same system tables and inputs on both sides.  Tolerances: local energies and
log ratios 1e-10 relative; symmetric-Metropolis VMC positions bit for bit
(every accept decision identical); DMC populations and branching identical.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import Oracle
from oracle.oracle import S_EL, S_LOGPSI

pytestmark = pytest.mark.gpu

SYSTEMS = ["exciton", "heg10", "crystal16", "heg42", "dipoles16", "heg10t", "heg10bf"]


def walkers(setup, capacity):
    import alea_b200
    return alea_b200.Walkers(setup, capacity=capacity)


def rel(a, b, floor=1e-12):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


@pytest.mark.parametrize("name", SYSTEMS)
def test_evaluate_matches_oracle(name):
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    o = Oracle(setup)
    o.init(pos)
    g = walkers(setup, 8)
    g.upload(pos)
    d = g.download()
    assert rel(d["local_energy"], o.scalar(S_EL)[:4]) < 1e-10
    assert rel(d["log_psi"], o.scalar(S_LOGPSI)[:4], floor=1.0) < 1e-10
    scale = max(1.0, np.abs(o.grad()[:4]).max())
    assert np.max(np.abs(d["grad"] - o.grad()[:4])) < 1e-10 * scale
    lscale = max(1.0, np.abs(o.lap()[:4]).max())
    assert np.max(np.abs(d["lap"] - o.lap()[:4])) < 1e-9 * lscale
    assert np.array_equal(d["positions"], o.pos()[:4])


@pytest.mark.parametrize("name", SYSTEMS)
def test_single_moves_match_oracle(name):
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    nw = pos.shape[0]
    o = Oracle(setup)
    o.init(pos)
    g = walkers(setup, 8)
    g.upload(pos)
    rng = np.random.default_rng(3)
    npart, dim = o.np, o.dim
    step = 0.3 if name == "exciton" else 8.0
    for it, p in enumerate([0, npart - 1, npart // 2, 1 % npart]):
        cur = g.download()["positions"].reshape(nw, npart, dim)[:, p, :]
        new = cur + step * rng.standard_normal(cur.shape)
        acc = np.array([(w + it) % 2 == 0 for w in range(nw)])
        lr, ph, ng, nl = g.move(p, new, acc)
        for w in range(nw):
            out = o.move(w, p, new[w], bool(acc[w]))
            assert abs(lr[w] - out[0]) < 1e-10 * max(1.0, abs(out[0]))
            if "twisted" in str(setup.get("slater", [{}])[0].get("type", "")):
                assert abs(np.angle(np.exp(1j * (ph[w] - out[1])))) < 1e-10   # continuous phase
            else:
                assert ph[w] == out[1]                                        # 0 or π
            assert np.max(np.abs(ng[w] - out[2:4])) < 1e-9 * max(1.0, np.abs(out[2:4]).max())
            assert np.max(np.abs(nl[w] - out[4:6])) < 1e-9 * max(1.0, np.abs(out[4:6]).max())
    g.measure()
    d = g.download()
    for w in range(nw):
        o.measure(w)
    assert np.array_equal(d["positions"], o.pos()[:nw])
    assert rel(d["local_energy"], o.scalar(S_EL)[:nw]) < 1e-10


@pytest.mark.parametrize("name,drift", [("exciton", False), ("heg10", False), ("heg10", True),
                                        ("crystal16", False), ("heg42", False), ("dipoles16", False),
                                        ("dipoles16", True), ("heg10t", False), ("heg10t", True),
                                        ("heg10bf", False), ("heg10bf", True)])
def test_vmc_steps_match_oracle(name, drift):
    import alea_b200
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    nw = pos.shape[0]
    tau = {"exciton": 0.05, "heg10": 225.0, "crystal16": 400.0, "heg42": 225.0,
           "dipoles16": 0.0003, "heg10t": 225.0, "heg10bf": 225.0}[name]
    n_steps, n_sub, seed = 4, 2, 21
    o = Oracle(setup)
    o.init(pos)
    el_o, st_o = o.vmc(nw, seed, 0, 1, n_steps, n_sub, tau, drift=drift)
    g = walkers(setup, nw)
    g.upload(pos)
    g.set_streams(seed, alea_b200.STREAM_VMC, nw)
    acc = 0
    for s in range(n_steps):
        st = g.vmc_step(tau, n_sub, drift)
        acc += st.n_accepted
        assert rel(g.download()["local_energy"], el_o[s]) < 1e-10
    assert acc == int(st_o[0])
    fin = g.download()["positions"]
    if drift:
        assert np.max(np.abs(fin - o.pos()[:nw])) < 1e-9 * np.abs(fin).max()
    else:
        assert np.array_equal(fin, o.pos()[:nw])


@pytest.mark.parametrize("name", ["exciton", "heg10", "dipoles16", "heg10t", "heg10bf"])
def test_dmc_run_matches_oracle(name):
    setup = golden(f"setup_{name}.json")
    r = golden(f"dmc_{name}.json")
    p = r["params"]
    nw = p["nw"]
    pos = np.array(r["initial_positions"])
    o = Oracle(setup)
    o.init(pos, capacity=4 * nw + 4)
    tr = o.dmc(nw, p["seed"], p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], target=nw)
    g = walkers(setup, 4 * nw + 4)
    g.upload(pos)
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw,
                            p["seed"], target=nw)
    n_eq = p["eq"] * p["steps"]
    ref_blocks = [tr[n_eq + b * p["steps"]: n_eq + (b + 1) * p["steps"], 1].sum() /
                  tr[n_eq + b * p["steps"]: n_eq + (b + 1) * p["steps"], 2].sum()
                  for b in range(p["acc"])]
    assert rel(blocks, ref_blocks) < 1e-10
    assert g.nw == o.nw                       # identical branching history
    assert rel(g.download()["local_energy"], o.scalar(S_EL)[: o.nw]) < 1e-9


def test_exciton_exact_energy_zero_variance():
    import alea_b200
    setup = golden("setup_exciton.json")
    pos = np.array(golden("eval_exciton.json")["positions"])
    pos = np.concatenate([pos] * 8)
    g = walkers(setup, len(pos))
    g.upload(pos)
    res, blocks = g.vmc_run(1, 4, 5, 2, 0.05, len(pos), 42)
    assert abs(res.energy + 1.0) < 1e-12
    assert res.variance < 1e-20
    assert 0.5 < res.acceptance < 1.0


@pytest.mark.gpu
def test_ewald_madelung_on_device():
    """Square-lattice Madelung constant from the device Ewald sum (reference
    known answer 1.6155426267, tests/test_ewald.cpp:212-225), equal to the
    oracle's to 1e-10."""
    import alea_b200
    from alea_b200 import setup as S
    from oracle import Oracle
    s = S.charges2d([2.0, 0.0, 0.0, 2.0], [2, 2], [1.0, -1.0], ewald_tol=1e-8)
    pos = np.array([[0.0, 0.0, 1.0, 1.0, 1.0, 0.0, 0.0, 1.0]])
    g = alea_b200.Walkers(s.desc, capacity=1)
    g.upload(pos)
    e_dev = g.download()["local_energy"][0]
    o = Oracle(s.desc)
    o.init(pos)
    assert abs(e_dev - o.measure(0)) < 1e-10 * abs(e_dev)
    assert -2.0 * e_dev / 4.0 == pytest.approx(1.6155426267, abs=1e-6)


@pytest.mark.gpu
def test_dmc_energy_agrees_with_reference_statistically():
    """A long device DMC run (independent seed and start) against the compiled
    reference's DMC on the same system and parameters: the block-averaged
    energies agree within 2 combined standard errors."""
    import alea_b200
    from alea_b200 import setup as S
    ref = golden("dmcstat_heg10.json")
    p = ref["params"]
    desc = golden("setup_heg10.json")
    start = S.heg2d(5, 5, 30.0).positions(777, p["nw"])
    g = alea_b200.Walkers(desc, capacity=2 * p["nw"] + 2)
    g.upload(start)
    res, blocks = g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], p["threads"],
                            seed=778, target=p["nw"], generations=10.0)
    assert len(blocks) == p["acc"] and np.all(np.isfinite(blocks))
    sigma = float(np.hypot(res.energy_error, ref["energy_error"]))
    assert res.energy_error > 0 and abs(res.energy - ref["energy"]) < 2.0 * sigma, \
        (res.energy, res.energy_error, ref["energy"], ref["energy_error"])


@pytest.mark.gpu
def test_twisted_phase_planes_match_oracle():
    """Complex determinant: phase part of ∇ln ψ, ∂²ln ψ and Im E_L after a
    full evaluation and after VMC steps (Sherman-Morrison updates)."""
    import alea_b200
    from oracle.oracle import S_ELI
    setup = golden("setup_heg10t.json")
    pos = np.array(golden("eval_heg10t.json")["positions"])
    nw = pos.shape[0]
    o = Oracle(setup)
    o.init(pos)
    g = walkers(setup, nw)
    g.upload(pos)
    ph = g.download_phase()
    scale = np.abs(o.phase_lap()[:nw]).max()
    assert np.max(np.abs(ph["phase_grad"] - o.phase_grad()[:nw])) < 1e-10 * scale
    assert np.max(np.abs(ph["phase_lap"] - o.phase_lap()[:nw])) < 1e-10 * scale
    assert np.max(np.abs(ph["local_energy_imag"] - o.scalar(S_ELI)[:nw])) < 1e-12
    el_o, _ = o.vmc(nw, 7, 0, 1, 3, 2, 225.0)
    g.set_streams(7, alea_b200.STREAM_VMC, nw)
    for _ in range(3):
        g.vmc_step(225.0, 2, False)
    ph = g.download_phase()
    assert np.max(np.abs(ph["phase_grad"] - o.phase_grad()[:nw])) < 1e-9 * scale
    assert np.max(np.abs(ph["local_energy_imag"] - o.scalar(S_ELI)[:nw])) < 1e-10
    assert rel(g.download()["local_energy"], el_o[-1]) < 1e-10


@pytest.mark.gpu
def test_free_twisted_determinant_kinetic_energy_on_device():
    """Twisted plane waves alone: E_L = Σ |k + θ|²/2 for every walker."""
    s = golden("setup_heg10t.json")
    free = {k: v for k, v in s.items() if k not in ("pade", "ewald")}
    pos = np.array(golden("eval_heg10t.json")["positions"])
    g = walkers(free, len(pos))
    g.upload(pos)
    q = np.concatenate([np.array(b["q"]) for b in s["slater"]])
    exact = 0.5 * np.sum(q * q)
    assert np.max(np.abs(g.download()["local_energy"] - exact)) < 1e-12 * abs(exact) + 1e-15


def _twisted42(nw):
    """The 21 + 21 electron gas at r_s = 30 and twist (1/8, 3/8): a complex
    determinant of the serving mix's size, with walkers from its own sampler."""
    from alea_b200 import setup as S
    st = S.heg2d_twisted(21, 21, 30.0, (0.125, 0.375))
    return st.desc, st.positions(4242, nw)


def _dipoles256(nw):
    """256 dipolar bosons of the serving mix (Jastrow-only, one-warp body
    for 65 to 256 particles)."""
    from alea_b200 import setup as S
    st = S.dipoles2d(256, 0.0353, 1.0, 3.0, 0.0459)
    return st.desc, st.positions(4242, nw)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["heg42", "crystal16", "dipoles16", "heg10t", "heg42t", "dipoles256"])
def test_one_warp_sweep_matches_generic_sweep(name, monkeypatch):
    """The one-warp sweeps (taken by 32-thread walkers of at most 64
    particles, real or complex determinants, and by Jastrow-only systems of
    65 to 256 particles) and the generic CTA sweep
    (ALEA_GPU_SWEEP=generic) on the same walkers and random streams: VMC
    positions bit for bit; after drift VMC and DMC advances, positions to
    1e-9 and E_L, Im E_L, weights, ln ψ to 1e-10."""
    import alea_b200
    if name == "heg42t":
        setup, pos = _twisted42(64)
    elif name == "dipoles256":
        setup, pos = _dipoles256(32)
    else:
        setup = golden(f"setup_{name}.json")
        pos = np.array(golden(f"eval_{name}.json")["positions"])
    nw = pos.shape[0]
    tau = {"heg42": 225.0, "crystal16": 400.0, "dipoles16": 0.0003, "heg10t": 225.0, "heg42t": 225.0,
           "dipoles256": 0.0003}[name]
    dtau = {"heg42": 0.5, "crystal16": 1.0, "dipoles16": 1e-5, "heg10t": 0.5, "heg42t": 0.5, "dipoles256": 1e-5}[name]
    out = []
    for mode in ("generic", "fast"):
        if mode == "generic":
            monkeypatch.setenv("ALEA_GPU_SWEEP", "generic")
        else:
            monkeypatch.delenv("ALEA_GPU_SWEEP", raising=False)
        g = walkers(setup, nw)
        g.upload(pos)
        g.set_streams(17, alea_b200.STREAM_VMC, nw)
        g.vmc_step(tau, 2, False)
        vmc_pos = g.download()["positions"]
        g.vmc_step(dtau, 2, True)
        g.set_streams(17, alea_b200.STREAM_DMC, nw)
        el = g.download()["local_energy"]
        e0 = float(np.mean(el))
        g.dmc_advance(dtau, 1, e0, e0, 10.0, 15.0)
        g.dmc_advance(dtau, 1, e0, e0, 10.0, 15.0)
        d = g.download()
        if name.endswith("t"):
            d.update(g.download_phase())
        out.append((vmc_pos, d))
        g.close()
    (vp_g, d_g), (vp_f, d_f) = out
    assert np.array_equal(vp_g, vp_f)
    assert np.max(np.abs(d_f["positions"] - d_g["positions"])) < 1e-9 * np.abs(d_g["positions"]).max()
    assert rel(d_f["local_energy"], d_g["local_energy"]) < 1e-10
    if name.endswith("t"):
        scale = np.abs(d_g["local_energy"]).max()
        assert np.max(np.abs(d_f["local_energy_imag"] - d_g["local_energy_imag"])) < 1e-10 * scale
        assert np.max(np.abs(d_f["phase_grad"] - d_g["phase_grad"])) < 1e-9 * np.abs(d_g["phase_grad"]).max()
    assert rel(d_f["log_psi"], d_g["log_psi"], floor=1.0) < 1e-10
    assert rel(d_f["weights"], d_g["weights"]) < 1e-10


def test_split_move_and_multi_step_entry_points_equal_the_fused_ones():
    """alea_gpu_propose / ratio / commit give alea_gpu_move's results bit for
    bit; alea_gpu_local_energy is measure + E_L; vmc_steps / dmc_steps equal
    their step loops (same streams, same walkers)."""
    import ctypes
    import alea_b200
    from alea_b200 import _capi
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"])
    nw = pos.shape[0]
    a, b = walkers(setup, 8), walkers(setup, 8)
    a.upload(pos)
    b.upload(pos)
    lib = _capi.load()
    dp = lambda x: x.ctypes.data_as(_capi.c_dp)
    rng = np.random.default_rng(5)
    for p in (0, 7, 3):
        new = np.ascontiguousarray((a.download()["positions"].reshape(nw, -1, 2)[:, p, :] +
                                    rng.normal(0, 8.0, (nw, 2))).T)
        acc = np.array([1, 0, 1, 1], dtype=np.uint8)
        lr_a, ph_a, g_a, l_a = a.move(p, new.T, acc)
        lr_b, ph_b = np.zeros(nw), np.zeros(nw)
        g_b, l_b = np.zeros(2 * nw), np.zeros(2 * nw)
        assert lib.alea_gpu_propose(b.ctx, p, dp(new)) == 0
        assert lib.alea_gpu_ratio(b.ctx, p, dp(lr_b), dp(ph_b), dp(g_b), dp(l_b)) == 0
        assert lib.alea_gpu_commit(b.ctx, p, acc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))) == 0
        assert np.array_equal(lr_a, lr_b) and np.array_equal(ph_a, ph_b)
        assert np.array_equal(g_a, g_b.reshape(2, nw).T) and np.array_equal(l_a, l_b.reshape(2, nw).T)
        assert lib.alea_gpu_commit(b.ctx, p, acc.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))) != 0
    el = np.zeros(nw)
    assert lib.alea_gpu_local_energy(b.ctx, dp(el)) == 0
    a.measure()
    assert np.array_equal(el, a.download()["local_energy"])
    for g in (a, b):
        g.set_streams(4, alea_b200.STREAM_VMC, nw)
    tot = [a.vmc_step(225.0, 1) for _ in range(3)]
    st = _capi.StepStats()
    prm = _capi.VmcParams(225.0, 1, 0)
    assert lib.alea_gpu_vmc_steps(b.ctx, ctypes.byref(prm), 3, ctypes.byref(st)) == 0
    assert st.n_accepted == sum(t.n_accepted for t in tot)
    assert np.array_equal(a.download()["positions"], b.download()["positions"])


def test_dmc_steps_equal_the_advance_branch_loop():
    import ctypes
    import alea_b200
    from alea_b200 import _capi
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"])
    nw = pos.shape[0]
    a, b = walkers(setup, 4 * nw + 4), walkers(setup, 4 * nw + 4)
    lib = _capi.load()
    for g in (a, b):
        g.upload(pos)
        assert lib.alea_gpu_set_rng_streams(g.ctx, ctypes.c_uint64(8), ctypes.c_uint64(alea_b200.STREAM_DMC), nw) == 0
    el0 = float(np.mean(a.download()["local_energy"]))
    prm = _capi.DmcParams(2.0, 1, el0, el0, np.inf, np.inf)
    sa = np.array([1, 2, 3, 4], dtype=np.uint64)
    sb = sa.copy()
    tot = 0
    for _ in range(3):
        st = a.dmc_advance(2.0, 1, el0, el0, np.inf, np.inf)
        a.dmc_branch(sa, nw)
        tot += st.n_accepted
    st = _capi.StepStats()
    assert lib.alea_gpu_dmc_steps(b.ctx, ctypes.byref(prm), 3, sb.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                  nw, ctypes.byref(st)) == 0
    assert st.n_accepted == tot and st.n_walkers == a.nw and np.array_equal(sa, sb)
    assert np.array_equal(a.download()["positions"], b.download()["positions"])
