"""The oracle restatement pinned against the reference (CPU only).

The expected values are the reference's own outputs: its xoshiro256++
known-answer test (tests/test_xoshiro_random.cpp:39-50 of the reference) and
golden fixtures produced by running the reference's VMC/DMC drivers and
components (tests/golden/make_fixtures.py).
"""
import numpy as np
import pytest

from conftest import golden
from oracle import Oracle
from oracle.oracle import S_EL, S_LOGPSI, load_oracle_lib

SYSTEMS = ["exciton", "heg10", "crystal16", "heg42", "dipoles16", "heg10t", "heg10bf", "crystal120"]


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-12)))


def test_xoshiro_known_answers():
    import ctypes
    lib = load_oracle_lib()
    state = (ctypes.c_uint64 * 4)(1, 2, 3, 4)
    out = (ctypes.c_uint64 * 10)()
    lib.o_xoshiro_raw(state, 10, out)
    assert list(out) == [41943041, 58720359, 3588806011781223, 3591011842654386,
                         9228616714210784205, 9973669472204895162, 14011001112246962877,
                         12406186145184390807, 15849039046786891736, 10450023813501588000]


def test_stream_seed_and_ziggurat():
    import ctypes
    lib = load_oracle_lib()
    # splitmix64 of 0 and the hashed stream seed are fixed bijections
    assert lib.o_splitmix64(0) == 0xE220A8397B1DCDAF
    a = lib.o_stream_seed(42, 0x766D632D74687264, 3)
    b = lib.o_stream_seed(42, 0x766D632D74687264, 4)
    assert a != b
    k = (ctypes.c_uint64 * 256)()
    w = (ctypes.c_double * 256)()
    f = (ctypes.c_double * 256)()
    r = ctypes.c_double()
    lib.o_ziggurat_tables(k, w, f, ctypes.byref(r))
    # the tail start agrees with Marsaglia & Tsang's 3.6541528853610088 to 1e-15
    assert abs(r.value - 3.6541528853610088) < 1e-14
    assert k[1] == 0 and f[0] == 1.0
    g = np.zeros(200000)
    lib.o_rng_draws(7, len(g), 1, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    assert abs(g.mean()) < 0.01 and abs(g.var() - 1.0) < 0.01


@pytest.mark.parametrize("name", SYSTEMS)
def test_oracle_evaluate_matches_reference(name):
    setup = golden(f"setup_{name}.json")
    ev = golden(f"eval_{name}.json")
    o = Oracle(setup)
    o.init(np.array(ev["positions"]))
    lp = o.scalar(S_LOGPSI)[:4]
    el = o.scalar(S_EL)[:4]
    # ln|psi| relative to walker 0 (its normalisation is not physical)
    ref_lp = np.array(ev["log_psi"])
    assert np.max(np.abs((lp - lp[0]) - (ref_lp - ref_lp[0]))) < 1e-9 * max(1.0, np.abs(ref_lp).max())
    assert rel(el, ev["local_energy"]) < 1e-10
    n = o.np * o.dim
    g_ref = np.array(ev["grad"]).reshape(n, -1).T
    assert np.max(np.abs(o.grad()[:4] - g_ref)) < 1e-9 * max(1.0, np.abs(g_ref).max())


@pytest.mark.parametrize("name", ["exciton", "heg10", "heg10_drift", "crystal16", "dipoles16",
                                  "heg10t", "heg10t_drift", "heg10bf", "heg10bf_drift", "crystal120",
                                  "heg42_crowd"])
def test_oracle_vmc_matches_reference(name):
    r = golden(f"vmc_{name}.json")
    p = r["params"]
    o = Oracle(golden(f"setup_{r['system']}.json"))
    o.init(np.array(r["initial_positions"]))
    T = p.get("threads", p["nw"])
    el, st = o.vmc(T, p["seed"], p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"],
                   drift=bool(p.get("drift", 0)))
    n_eq_steps = p["eq"] * p["steps"]
    # thread t's list: its contiguous walkers' E_L, step after step
    nw = p["nw"]
    lo = [t * (nw // T) + min(t, nw % T) for t in range(T + 1)]
    mine = [el[n_eq_steps:, lo[t]:lo[t + 1]].ravel() for t in range(T)]
    for t in range(T):
        assert rel(mine[t], r["thread_local_energy"][t]) < 1e-10
    assert st[0] / st[1] == pytest.approx(r["acceptance"], abs=0, rel=1e-15)
    fp = np.array(r["final_positions"]).reshape(p["nw"], -1)
    if p.get("drift", 0):
        assert np.max(np.abs(o.pos()[: p["nw"]] - fp)) < 1e-9 * np.abs(fp).max()
    else:
        # symmetric Metropolis moves: the same decisions give bitwise positions
        assert np.array_equal(o.pos()[: p["nw"]], fp)


@pytest.mark.parametrize("name", ["exciton", "heg10", "dipoles16", "heg10t", "heg10bf", "heg42",
                                  "heg42_crowd"])
def test_oracle_dmc_matches_reference(name):
    r = golden(f"dmc_{name}.json")
    p = r["params"]
    o = Oracle(golden(f"setup_{r['system']}.json"))
    o.init(np.array(r["initial_positions"]), capacity=4 * p["nw"] + 4)
    tr = o.dmc(p.get("threads", p["nw"]), p["seed"], p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"],
               target=p["nw"])
    n_eq_steps = p["eq"] * p["steps"]
    pops_ref = [len(x) for x in r["local_energy"]]
    assert tr[n_eq_steps:, 0].astype(int).tolist() == pops_ref      # branching counts
    assert rel(tr[n_eq_steps:, 2], r["weight_sum"]) < 1e-12
    assert rel(tr[n_eq_steps:, 1], r["weighted_energy_sum"]) < 1e-10


def test_exciton_exact_zero_variance():
    s = golden("setup_exciton.json")
    ev = golden("eval_exciton.json")
    o = Oracle(s)
    o.init(np.array(ev["positions"]))
    el, _ = o.vmc(4, 1, 0, 3, 5, 2, 0.05)
    assert np.max(np.abs(el + 1.0)) < 1e-12


def test_oracle_twisted_phase_planes_match_reference():
    """Complex determinant: the phase part of ∇ln ψ and ∂²ln ψ and Im E_L."""
    from oracle.oracle import S_ELI
    ev = golden("eval_heg10t.json")
    o = Oracle(golden("setup_heg10t.json"))
    o.init(np.array(ev["positions"]))
    n = o.np * o.dim
    for mine, key in ((o.phase_grad(), "phase_grad"), (o.phase_lap(), "phase_lap")):
        ref = np.array(ev[key]).reshape(n, -1).T
        assert np.max(np.abs(mine[:4] - ref)) < 1e-10 * max(1.0, np.abs(ref).max())
    assert np.max(np.abs(o.scalar(S_ELI)[:4] - np.array(ev["local_energy_imag"]))) < 1e-12


def test_oracle_free_twisted_determinant_kinetic_energy():
    """A determinant of twisted plane waves alone is an eigenstate of the
    kinetic energy: E_L = Σ |k + θ|²/2 for every configuration
    (complex_orbital_set.h kinetic_energy_sum)."""
    s = golden("setup_heg10t.json")
    free = {k: v for k, v in s.items() if k not in ("pade", "ewald")}
    ev = golden("eval_heg10t.json")
    o = Oracle(free)
    o.init(np.array(ev["positions"]))
    q = np.concatenate([np.array(b["q"]) for b in s["slater"]])
    exact = 0.5 * np.sum(q * q)
    assert np.max(np.abs(o.scalar(S_EL)[:4] - exact)) < 1e-12 * abs(exact) + 1e-15
