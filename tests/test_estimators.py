"""Observable estimators: g(r), density grid, S(k) and ρ_g(k).

CPU: the oracle restatement against the compiled reference's estimators on
the golden configurations (est_<name>.json), and the package's host-side
finalize on the oracle's block estimates.  GPU (through the C ABI): the
device's block estimates against the oracle's on the same configurations and
weights (dyadic weights: every histogram bin is an exact sum, so g(r) and
density blocks agree bit for bit), and whole VMC / DMC runs with estimators
against the reference drivers' series.
"""
import numpy as np
import pytest

from conftest import golden
from oracle import Oracle
from oracle import estimators as OE

SYSTEMS = ["heg10", "dipoles16"]


def oracle_estimators(o, est):
    out = []
    if est.get("gofr_bins"):
        out.append(OE.Gofr(o, est["gofr_rmax"], est["gofr_bins"]))
    if est.get("dens_bins"):
        out.append(OE.Density(o, est["dens_rmax"], est["dens_bins"], bool(est.get("dens_pp", 0))))
    if est.get("sofk_kmax"):
        out.append(OE.Sofk(o, est["sofk_kmax"]))
    return out


def run_oracle(name):
    r = golden(f"est_{name}.json")
    o = Oracle(golden(f"setup_{name}.json"))
    ests = oracle_estimators(o, r["est"])
    confs = r["configurations"]
    steps = r["params"]["steps"]
    for b in range(r["params"]["acc"]):
        for e in ests:
            e.start_block()
        for c in confs[b * steps:(b + 1) * steps]:
            for e in ests:
                e.accumulate(np.array(c["positions"]), np.array(c["weights"]))
        for e in ests:
            e.stop_block()
    return r, ests


def by_k(series, kx, ky):
    """Series values keyed by the rounded k vector (the reference sorts k by
    |k| with std::sort, which leaves the order inside a shell unspecified)."""
    return {(round(x, 9), round(y, 9)): v for x, y, v in zip(kx, ky, series)}


def compare(out, ref, tol, skip=()):
    for k, v in out.items():
        if k in skip:
            continue
        rv = np.array(ref[k], dtype=float)
        v = np.asarray(v, dtype=float)
        if k.startswith("rhok") or (k.startswith("sofk") and k.rsplit("_", 1)[-1] in ("kx", "ky", "shell")):
            a = by_k(v, out["sofk_kx"], out["sofk_ky"])
            b = by_k(rv, ref["sofk_kx"], ref["sofk_ky"])
            assert a.keys() == b.keys(), k
            v = np.array([a[q] for q in sorted(a)])
            rv = np.array([b[q] for q in sorted(b)])
        scale = max(np.abs(rv).max(), 1e-300)
        assert v.shape == rv.shape, k
        assert np.max(np.abs(v - rv)) <= tol * scale, (k, np.max(np.abs(v - rv)) / scale)


@pytest.mark.parametrize("name", SYSTEMS)
def test_oracle_estimators_match_reference(name):
    r, ests = run_oracle(name)
    out = {}
    for e in ests:
        out.update(e.finalize())
    assert set(out) <= set(r["estimators"])
    compare(out, r["estimators"], 1e-13)


@pytest.mark.parametrize("name", SYSTEMS)
def test_host_finalize_matches_reference(name):
    """alea_b200.estimators on the oracle's block estimates gives the
    reference's series (the package's host logic, no GPU)."""
    from alea_b200 import estimators as E
    r, ests = run_oracle(name)
    setup = golden(f"setup_{name}.json")
    groups = setup["groups"]
    out = {}
    for e in ests:
        if isinstance(e, OE.Gofr):
            out.update(E.finalize_gofr(np.array(e.history), groups, e.rmax, e.n_bins, e.volume))
        elif isinstance(e, OE.Density):
            out.update(E.finalize_density(np.array([e.history]), groups, e.n_bins, e.pp))
        else:
            blocks = np.array([np.concatenate([s, re, im]) for s, re, im in
                               zip(e.hist_s, e.hist_re, e.hist_im)])
            out.update(E.finalize_sofk(blocks, groups, e.k))
    compare(out, r["estimators"], 1e-13)


def test_density_chain_merge_matches_clone_collect():
    """Chains merged in order (Chan et al.) equal the reference's clone
    collect: two oracle Density clones, one per half of the blocks."""
    from alea_b200 import estimators as E
    name = "heg10"
    r = golden(f"est_{name}.json")
    o = Oracle(golden(f"setup_{name}.json"))
    a, b = OE.Density(o, 84.0, 8), OE.Density(o, 84.0, 8)
    for i, c in enumerate(r["configurations"]):
        e = a if i < 3 else b
        e.start_block()
        e.accumulate(np.array(c["positions"]), np.array(c["weights"]))
        e.stop_block()
    chains = np.array([a.history, b.history])
    a.collect(b)
    want = a.finalize()
    got = E.finalize_density(chains, golden(f"setup_{name}.json")["groups"], 8)
    for k in want:
        assert np.allclose(got[k], want[k], rtol=1e-13, atol=1e-300), k


# ───────────────────────── device ───────────────────────────────────────

def device_estimators(g, est):
    ids = {}
    if est.get("gofr_bins"):
        ids["gofr"] = g.add_estimator("gofr", n_bins=est["gofr_bins"], rmax=est["gofr_rmax"])
    if est.get("dens_bins"):
        ids["density"] = g.add_estimator("density", n_bins=est["dens_bins"], rmax=est["dens_rmax"],
                                         per_particle=bool(est.get("dens_pp", 0)))
    if est.get("sofk_kmax"):
        ids["sofk"] = g.add_estimator("sofk", kmax=est["sofk_kmax"])
    return ids


@pytest.mark.gpu
@pytest.mark.parametrize("name", SYSTEMS)
def test_device_blocks_match_oracle(name):
    import alea_b200
    r, ests = run_oracle(name)
    setup = golden(f"setup_{name}.json")
    npart, dim = int(setup["np"]), int(setup["dim"])
    nw = r["params"]["nw"]
    g = alea_b200.Walkers(setup, capacity=nw)
    ids = device_estimators(g, r["est"])
    steps = r["params"]["steps"]
    confs = r["configurations"]
    for b in range(r["params"]["acc"]):
        g.estimators_start_block()
        for c in confs[b * steps:(b + 1) * steps]:
            soa = np.array(c["positions"]).reshape(npart * dim, nw)
            g.upload(soa.T.reshape(nw, npart, dim))
            g.estimators_accumulate(np.array(c["weights"]))
        g.estimators_stop_block()
    for e in ests:
        if isinstance(e, OE.Gofr):
            dev = g.estimator_blocks(ids["gofr"])[0]
            assert np.array_equal(dev, np.array(e.history))
        elif isinstance(e, OE.Density):
            dev = g.estimator_blocks(ids["density"])[0]
            assert np.array_equal(dev, np.array(e.history))
        else:
            dev = g.estimator_blocks(ids["sofk"])[0]
            kv = g.estimator_kvectors(ids["sofk"])
            assert np.array_equal(kv["n1"], e.k["n1"]) and np.array_equal(kv["n2"], e.k["n2"])
            want = np.array([np.concatenate([s, re, im]) for s, re, im in zip(e.hist_s, e.hist_re, e.hist_im)])
            assert np.max(np.abs(dev - want)) <= 1e-12 * np.abs(want).max()
    out = {}
    for k, i in ids.items():
        out.update(g.estimator_results(i))
    compare(out, r["estimators"], 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SYSTEMS + ["crystal16"])
def test_vmc_run_estimators_match_reference(name):
    """VMC::run with the estimators attached, one stream (and estimator
    clone) per walker: symmetric-Metropolis positions are bit-identical, so
    every histogram is too."""
    import alea_b200
    ref = golden(f"est_vmc_{name}.json")
    p = ref["params"]
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"vmc_{name}.json")["initial_positions"])
    nw = p["nw"]
    g = alea_b200.Walkers(setup, capacity=nw)
    g.upload(pos)
    ids = device_estimators(g, ref["est"])
    g.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"])
    assert np.array_equal(g.download()["positions"].ravel(), np.array(ref["final_positions"]))
    d = g.estimator_desc(ids["gofr"])
    assert d.n_chains == nw and d.n_blocks == p["acc"]
    out = {}
    for k, i in ids.items():
        out.update(g.estimator_results(i))
    compare(out, ref["estimators"], 1e-12)


@pytest.mark.gpu
def test_dmc_run_estimators_match_reference():
    """DMC::run's mixed estimators (population before each branch, DMC
    weights): same populations as the reference, positions equal to
    rounding, so the series agree to 1e-9."""
    import alea_b200
    name = "heg10"
    ref = golden(f"est_dmc_{name}.json")
    p = ref["params"]
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"dmc_{name}.json")["initial_positions"])
    nw = p["nw"]
    g = alea_b200.Walkers(setup, capacity=4 * nw + 4)
    g.upload(pos)
    ids = device_estimators(g, ref["est"])
    g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"], target=nw)
    d = g.estimator_desc(ids["density"])
    assert d.n_chains == 1 and d.n_blocks == p["acc"]
    out = {}
    for k, i in ids.items():
        out.update(g.estimator_results(i))
    compare(out, ref["estimators"], 1e-9)


@pytest.mark.gpu
def test_estimator_errors():
    import alea_b200
    setup = golden("setup_heg10.json")
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(np.array(golden("eval_heg10.json")["positions"]))
    with pytest.raises(alea_b200.AleaGpuError):
        g.add_estimator("gofr", n_bins=10, rmax=1e4)        # beyond the Wigner-Seitz inradius
    with pytest.raises(alea_b200.AleaGpuError):
        g.add_estimator("sofk", kmax=1e-6)                  # no k below kmax
    g.add_estimator("gofr", n_bins=10, rmax=50.0)
    g.estimators_accumulate(chains=2)
    with pytest.raises(alea_b200.AleaGpuError):
        g.estimators_accumulate(chains=1)                   # chain count fixed until a reset
    g.estimators_reset()
    g.estimators_accumulate(chains=1)
    g.estimators_stop_block()
    assert g.estimator_desc(0).n_blocks == 1


@pytest.mark.gpu
def test_ragged_chains_match_per_chain_oracle():
    """Chains that do not divide the population (10 walkers in 3 chains of
    4, 3, 3, VMC's even split): every chain's block equals the oracle run on
    that chain's walkers alone, bit for bit (dyadic weights)."""
    import alea_b200
    name = "heg10"
    r = golden(f"est_{name}.json")
    setup = golden(f"setup_{name}.json")
    confs = r["configurations"]
    npart = int(setup["np"])
    pos = np.concatenate([np.array(c["positions"]).reshape(npart * 2, -1).T for c in confs[:2]])[:10]
    wts = np.concatenate([np.array(c["weights"]) for c in confs[:2]])[:10]
    g = alea_b200.Walkers(setup, capacity=10)
    g.upload(pos.reshape(10, npart, 2))
    gid = g.add_estimator("gofr", n_bins=20, rmax=80.0)
    did = g.add_estimator("density", n_bins=8, rmax=84.0)
    g.estimators_accumulate(wts, chains=3)
    g.estimators_stop_block()
    o = Oracle(setup)
    starts = [0, 4, 7, 10]
    for t in range(3):
        sl = slice(starts[t], starts[t + 1])
        soa = np.ascontiguousarray(g.download()["positions"][sl].T)
        og, od = OE.Gofr(o, 80.0, 20), OE.Density(o, 84.0, 8)
        for e in (og, od):
            e.accumulate(soa, wts[sl])
            e.stop_block()
        assert np.array_equal(g.estimator_blocks(gid)[t, 0], og.history[0])
        assert np.array_equal(g.estimator_blocks(did)[t, 0], od.history[0])


@pytest.mark.gpu
def test_estimator_size_limits_are_refused():
    import alea_b200
    setup = golden("setup_heg10.json")
    g = alea_b200.Walkers(setup, capacity=8)
    g.upload(np.array(golden("eval_heg10.json")["positions"]))
    g.add_estimator("gofr", n_bins=6000, rmax=80.0)        # counters beyond one warp's shared memory
    with pytest.raises(alea_b200.AleaGpuError) as e:
        g.estimators_accumulate()
    assert e.value.code == 3
    g.clear_estimators()
    with pytest.raises(alea_b200.AleaGpuError):
        g.add_estimator("density", n_bins=5000)              # more than 4096 bins per axis
    g.add_estimator("gofr", n_bins=1, rmax=80.0)             # the smallest histogram
    g.estimators_accumulate()
    g.estimators_stop_block()
    assert g.estimator_blocks(0).shape == (1, 1, 3)


@pytest.mark.gpu
def test_per_particle_density_sums_to_group_density():
    """On a DMC run (non-dyadic weights, population changing at every
    branch) the per-particle series of each group add up to the group's
    density series, block by block (1e-12): the per-particle grids and the
    group grids bin the same walkers with the same weights."""
    import alea_b200
    setup = golden("setup_heg10.json")
    ref = golden("dmc_heg10.json")
    nw = len(ref["initial_positions"])
    g = alea_b200.Walkers(setup, capacity=4 * nw + 4)
    g.upload(np.array(ref["initial_positions"]))
    grp = g.add_estimator("density", n_bins=8, rmax=84.0)
    per = g.add_estimator("density", n_bins=8, rmax=84.0, per_particle=True)
    g.dmc_run(1, 3, 4, 1, 2.0, nw, 7, target=nw)
    a, b = g.estimator_blocks(grp), g.estimator_blocks(per)
    n_cells = 64
    assert a.shape[:2] == b.shape[:2] and a.shape[1] == 3
    for q, G in enumerate(setup["groups"]):
        want = a[..., q * n_cells:(q + 1) * n_cells]
        got = sum(b[..., p * n_cells:(p + 1) * n_cells] for p in range(G["first"], G["last"]))
        assert np.max(np.abs(got - want)) <= 1e-12 * np.abs(want).max()
