"""Packed VMC runs (alea_gpu_vmc_run_packed): the walkers of several
contexts with different systems, particle numbers and walker counts swept in
one launch per step.  Each run's result must be its alea_gpu_vmc_run result
on its own context (same streams, same walker arithmetic): energy, error and
acceptance equal, variance to 1e-12; and the same alone as in the mix.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

# system, walkers, tau: the one-warp bodies (real determinants, bosons;
# twisted = complex determinants) and the generic body (backflow)
MIX = [("heg10", 64, 225.0), ("crystal16", 40, 400.0), ("dipoles16", 24, 0.0003),
       ("heg10t", 48, 225.0), ("heg10bf", 32, 225.0)]


def _walkers(name, nw):
    import alea_b200
    desc = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    reps = -(-nw // len(pos))
    g = alea_b200.Walkers(desc, capacity=nw)
    g.upload(np.concatenate([pos] * reps)[:nw])
    return g


def _run(k):
    name, nw, tau = MIX[k]
    return dict(n_eq=1, n_acc=3, n_steps=2, n_substeps=2, tau=tau, streams=max(1, nw // 8), seed=100 + k)


def _same(a, b):
    assert a.energy == b.energy and a.energy_error == b.energy_error
    assert a.acceptance == b.acceptance
    assert a.variance == pytest.approx(b.variance, rel=1e-12, abs=1e-300)
    assert a.n_moves == b.n_moves and a.n_evaluations == b.n_evaluations and a.n_walkers == b.n_walkers


def test_packed_runs_equal_their_own_vmc_runs():
    import alea_b200
    alone = []
    for k, (name, nw, tau) in enumerate(MIX):
        g = _walkers(name, nw)
        r = _run(k)
        res, _ = g.vmc_run(r["n_eq"], r["n_acc"], r["n_steps"], r["n_substeps"], r["tau"], r["streams"], r["seed"])
        alone.append(res)
        g.close()
    gs = [_walkers(name, nw) for name, nw, _ in MIX]
    packed = alea_b200.vmc_run_packed(gs, [_run(k) for k in range(len(MIX))])
    for k, (res, status) in enumerate(packed):
        assert status == 0
        _same(res, alone[k])
    # the same run packed alone
    for k in (0, 3):
        name, nw, _ = MIX[k]
        g = _walkers(name, nw)
        (res, status), = alea_b200.vmc_run_packed([g], [_run(k)])
        assert status == 0
        _same(res, packed[k][0])
        g.close()
    for g in gs:
        g.close()


def test_packed_runs_of_uneven_length():
    """Runs that finish at different steps leave the packed launch; the others
    go on unchanged (a second packed call replays captured steps)."""
    import alea_b200
    runs = [dict(_run(0), n_acc=1), dict(_run(2), n_acc=4), dict(_run(3), n_acc=2)]
    names = [MIX[0], MIX[2], MIX[3]]
    ref = []
    for (name, nw, _), r in zip(names, runs):
        g = _walkers(name, nw)
        res, _ = g.vmc_run(r["n_eq"], r["n_acc"], r["n_steps"], r["n_substeps"], r["tau"], r["streams"], r["seed"])
        ref.append(res)
        g.close()
    for _ in range(2):
        gs = [_walkers(name, nw) for name, nw, _ in names]
        out = alea_b200.vmc_run_packed(gs, runs)
        for (res, status), want in zip(out, ref):
            assert status == 0
            _same(res, want)
        for g in gs:
            g.close()


def test_packed_jastrow_only_body_with_the_others():
    """The one-warp Jastrow-only body (256 dipolar bosons) packed beside the
    real and complex one-warp bodies: each run equals its own vmc_run."""
    import alea_b200
    from alea_b200 import setup as S
    dip = S.dipoles2d(256, 0.0353, 1.0, 3.0, 0.0459)
    dpos = dip.positions(71, 24)

    def dipoles():
        g = alea_b200.Walkers(dip.desc, capacity=len(dpos))
        g.upload(dpos)
        return g

    makers = [dipoles, lambda: _walkers("heg10", MIX[0][1]), lambda: _walkers("heg10t", MIX[3][1])]
    runs = [dict(n_eq=1, n_acc=2, n_steps=1, n_substeps=1, tau=0.0003, streams=3, seed=500), _run(0), _run(3)]
    alone = []
    for make, r in zip(makers, runs):
        g = make()
        res, _ = g.vmc_run(r["n_eq"], r["n_acc"], r["n_steps"], r["n_substeps"], r["tau"], r["streams"], r["seed"])
        alone.append(res)
        g.close()
    gs = [make() for make in makers]
    packed = alea_b200.vmc_run_packed(gs, runs)
    for (res, status), want in zip(packed, alone):
        assert status == 0
        _same(res, want)
    for g in gs:
        g.close()
    dip.close()
