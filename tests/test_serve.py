"""Serving (include/alea_gpu.h, serving): the twisted electron-gas builder the
serving mix draws from, and the job server on the device — a job's result is
the same alone and in a mix, queued jobs cancel, polls are bounded, and
admission refuses a job over the memory budget."""
import itertools

import numpy as np
import pytest

from alea_b200 import setup as S


def _twisted_q(L, n, tx, ty):
    """The n lowest |k + θ| of the square reciprocal lattice 2π/L Z², θ = t b."""
    b = 2.0 * np.pi / L
    ij = np.array(list(itertools.product(range(-12, 13), repeat=2)), dtype=float)
    q = (ij + [tx, ty]) * b
    q2 = np.sum(q * q, axis=1)
    order = np.argsort(q2, kind="stable")
    return q[order[:n]], q2[order[n]] - q2[order[n - 1]]


@pytest.mark.parametrize("n,twist", [(13, (0.125, 0.125)), (21, (0.125, 0.375)), (29, (0.375, 0.125)),
                                     (45, (0.625, 0.875))])
def test_twisted_shells_are_the_lowest_k_plus_theta(n, twist):
    s = S.heg2d_twisted(n, n, 30.0, twist)
    d = s.desc
    L = d["cell"]["vectors"][0]
    want, gap = _twisted_q(L, n, *twist)
    assert gap > 1e-9
    for blk in d["slater"]:
        assert blk["type"] == "twisted_plane_wave"
        got = np.array(blk["q"]).reshape(-1, 2)
        assert sorted(map(tuple, np.round(got, 12))) == sorted(map(tuple, np.round(want, 12)))
    s.close()


def test_twist_that_splits_a_shell_is_refused():
    with pytest.raises(ValueError, match="degenerate"):
        S.heg2d_twisted(13, 13, 30.0, (0.125, 0.375))


def test_integer_twist_is_the_real_closed_shell_gas():
    a = S.heg2d_twisted(21, 21, 30.0, (1.0, 0.0)).desc
    b = S.heg2d(21, 21, 30.0).desc
    assert a["slater"] == b["slater"]


# ─────────────────────────── device ─────────────────────────────────────

def _jobs():
    heg = S.heg2d(5, 5, 30.0)
    tw = S.heg2d_twisted(5, 5, 30.0, (0.125, 0.125))
    dip = S.dipoles2d(16, 10.0)
    return [(heg, 0, 225.0), (tw, 0, 225.0), (dip, 0, 0.0003), (heg, 1, 0.5)]


@pytest.mark.gpu
def test_served_job_is_the_same_alone_and_in_a_mix():
    import alea_b200
    jobs = _jobs()

    def submit(srv, k):
        st, mode, tau = jobs[k]
        pos = st.positions(100 + k, 64)
        return srv.submit(st.desc, pos, mode, 1, 3, 4, 1, tau, seed=7 + k)

    alone = []
    for k in range(len(jobs)):
        srv = alea_b200.Server(max_running=1)
        r = srv.poll(submit(srv, k), timeout_ms=120000)
        assert r is not None and r.status == 0
        alone.append(r.result)
        srv.close()
    srv = alea_b200.Server(max_running=4)
    ids = [submit(srv, k) for k in range(len(jobs))] + [submit(srv, k) for k in range(len(jobs))]
    mixed = [srv.poll(i, timeout_ms=120000) for i in ids]
    srv.close()
    for k, r in enumerate(mixed):
        assert r is not None and r.status == 0
        a = alone[k % len(jobs)]
        assert r.result.energy == a.energy and r.result.energy_error == a.energy_error
        assert r.result.acceptance == a.acceptance and r.result.n_moves == a.n_moves
        assert r.latency_ms >= r.run_ms > 0.0


@pytest.mark.gpu
def test_cancel_poll_timeout_and_admission():
    import alea_b200
    from alea_b200 import _capi
    st, mode, tau = _jobs()[0]
    pos = st.positions(3, 64)
    srv = alea_b200.Server(max_running=1)
    long_job = srv.submit(st.desc, pos, 0, 1, 400, 8, 1, tau, seed=1)
    queued = srv.submit(st.desc, pos, 0, 1, 1, 1, 1, tau, seed=2)
    assert srv.poll(long_job, timeout_ms=0) is None          # still running: no wait
    assert srv.cancel(queued)
    r = srv.poll(queued, timeout_ms=1000)
    assert r is not None and r.status == _capi.ERR_CANCELLED
    assert srv.cancel(long_job)                                # running: stops at its next step
    r = srv.poll(long_job, timeout_ms=60000)
    assert r is not None and r.status == _capi.ERR_CANCELLED
    assert not srv.cancel(long_job)                            # already finished
    srv.close()
    small = alea_b200.Server(hbm_budget_bytes=1 << 20, max_running=1)
    with pytest.raises(alea_b200.AleaGpuError):
        small.submit(st.desc, pos, 0, 1, 1, 1, 1, tau, seed=3)
    small.close()


@pytest.mark.gpu
def test_twisted_builder_evaluates_like_the_oracle():
    """A twisted electron gas from the host builder: device ln|ψ|, phase
    planes and E_L against the oracle on the same walkers (1e-10)."""
    import alea_b200
    from oracle import Oracle
    from oracle.oracle import S_EL, S_LOGPSI
    st = S.heg2d_twisted(5, 5, 30.0, (0.125, 0.125))
    pos = st.positions(11, 4)
    g = alea_b200.Walkers(st.desc, capacity=4)
    g.upload(pos)
    d = g.download()
    o = Oracle(st.desc)
    o.init(pos)
    el_o = o.scalar(S_EL)[:4]
    assert np.max(np.abs(d["local_energy"] - el_o) / np.abs(el_o)) < 1e-10
    assert np.max(np.abs(d["log_psi"] - o.scalar(S_LOGPSI)[:4])) < 1e-10 * max(1.0, np.abs(d["log_psi"]).max())
    ph = g.download_phase()
    assert np.max(np.abs(ph["phase_grad"] - o.phase_grad()[:4])) < 1e-10 * max(1.0, np.abs(o.phase_grad()).max())
    g.close()


@pytest.mark.gpu
def test_budget_of_one_job_runs_jobs_one_after_another():
    """A server whose memory budget holds exactly one job's footprint: two
    jobs in a row both run (the second is admitted only once the first's
    context has released its memory) and a polled job is forgotten."""
    import alea_b200
    st, mode, tau = _jobs()[0]
    pos = st.positions(5, 64)
    probe = alea_b200.Server(max_running=1)
    r = probe.poll(probe.submit(st.desc, pos, 0, 1, 1, 1, 1, tau, seed=1), timeout_ms=60000)
    probe.close()
    assert r is not None and r.status == 0 and r.footprint_bytes > 0
    srv = alea_b200.Server(hbm_budget_bytes=int(r.footprint_bytes), max_running=2)
    ids = [srv.submit(st.desc, pos, 0, 1, 2, 2, 1, tau, seed=2 + k) for k in range(2)]
    res = [srv.poll(i, timeout_ms=60000) for i in ids]
    assert all(x is not None and x.status == 0 for x in res)
    assert res[1].queue_ms >= res[0].run_ms * 0.5       # it waited for the first to finish
    with pytest.raises(alea_b200.AleaGpuError):
        srv.poll(ids[0], timeout_ms=0)                  # handed out once
    srv.close()


@pytest.mark.gpu
def test_packed_server_job_is_the_same_alone_in_a_mix_and_as_its_own_run():
    """A packed server steps every admitted VMC job together (one sweep launch
    per step for all of them): each job's result is bit for bit the same
    alone, in a mix of four kinds (plane-wave, twisted, dipolar and Gaussian
    systems, different walker counts) and as alea_gpu_vmc_run on its own
    context; a queued job can still be cancelled."""
    import alea_b200
    from alea_b200 import _capi
    heg = S.heg2d(5, 5, 30.0)
    tw = S.heg2d_twisted(5, 5, 30.0, (0.125, 0.125))
    dip = S.dipoles2d(16, 10.0)
    jobs = [(heg, 64, 225.0), (tw, 48, 225.0), (dip, 40, 0.0003), (heg, 24, 100.0)]

    def submit(srv, k):
        st, nw, tau = jobs[k]
        return srv.submit(st.desc, st.positions(300 + k, nw), 0, 1, 3, 2 + k, 1, tau, seed=17 + k,
                          n_streams=max(1, nw // 4))

    alone = []
    for k in range(len(jobs)):
        srv = alea_b200.Server(max_running=1, packed=True)
        r = srv.poll(submit(srv, k), timeout_ms=120000)
        assert r is not None and r.status == 0
        alone.append(r.result)
        srv.close()
        st, nw, tau = jobs[k]
        g = alea_b200.Walkers(st.desc, capacity=nw)
        g.upload(st.positions(300 + k, nw))
        own, _ = g.vmc_run(1, 3, 2 + k, 1, tau, max(1, nw // 4), 17 + k)
        assert own.energy == r.result.energy and own.energy_error == r.result.energy_error
        assert own.acceptance == r.result.acceptance and own.n_moves == r.result.n_moves
        g.close()
    srv = alea_b200.Server(max_running=1, packed=True)
    ids = [submit(srv, k % len(jobs)) for k in range(2 * len(jobs))]
    extra = submit(srv, 0)
    srv.cancel(extra)
    got = [srv.poll(i, timeout_ms=120000) for i in ids]
    r_extra = srv.poll(extra, timeout_ms=120000)
    srv.close()
    assert r_extra is not None and r_extra.status in (0, _capi.ERR_CANCELLED)
    for k, r in enumerate(got):
        assert r is not None and r.status == 0
        a = alone[k % len(jobs)]
        assert r.result.energy == a.energy and r.result.energy_error == a.energy_error
        assert r.result.acceptance == a.acceptance and r.result.n_moves == a.n_moves
