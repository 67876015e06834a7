"""Walker configurations out and in: checkpoint rows, seeding, stage carry-over.

CPU: the checkpoint file round trip and the reference's walkers_in checks
(src/qmc/app.cpp:834-866).  GPU (through the C ABI): final configurations of
a symmetric-Metropolis VMC run equal the reference's bit for bit; a DMC seeded
from them (carry_over_walkers, app.cpp:1078-1098) reproduces the reference's
populations and weighted energies; seeding cycles rows; the state-keeping
carry-over hands over the walkers' records unchanged.
"""
import numpy as np
import pytest

from conftest import golden


def test_checkpoint_round_trip_and_checks(tmp_path):
    from alea_b200 import checkpoint as C
    desc = golden("setup_heg10.json")
    rows = np.random.default_rng(1).uniform(-80, 80, size=(7, 10, 2))
    path = str(tmp_path / "wk.npz")
    C.write_walkers(path, rows, lattice=desc["cell"]["vectors"], tag="eq", blocks_done=12)
    wf = C.read_walkers(path)
    assert wf["nw"] == 7 and wf["np"] == 10 and wf["dim"] == 2
    assert np.array_equal(wf["positions"], rows) and wf["tag"] == "eq" and wf["blocks_done"] == 12
    C.check_compatible(wf, desc)
    with pytest.raises(C.CheckpointError):
        C.check_compatible(wf, golden("setup_heg42.json"))          # geometry mismatch
    other = dict(desc, cell=dict(desc["cell"], vectors=[v * 1.001 for v in desc["cell"]["vectors"]]))
    with pytest.raises(C.CheckpointError):
        C.check_compatible(wf, other)                                # different density
    C.write_walkers(path, rows)                                      # open-cell file into a periodic run
    with pytest.raises(C.CheckpointError):
        C.check_compatible(C.read_walkers(path), desc)
    with pytest.raises(C.CheckpointError):
        C.read_walkers(str(tmp_path / "missing.npz"))


def chain_blocks(r, p):
    n_eq = p["dmc_eq"] * p["dmc_steps"]
    w, we = r["weight_sum"], r["weighted_energy_sum"]
    # the measure hook runs in accumulation steps only
    assert len(w) == p["dmc_acc"] * p["dmc_steps"]
    return [sum(we[b * p["dmc_steps"]:(b + 1) * p["dmc_steps"]]) / sum(w[b * p["dmc_steps"]:(b + 1) * p["dmc_steps"]])
            for b in range(p["dmc_acc"])], n_eq


@pytest.mark.gpu
def test_vmc_to_dmc_chain_matches_reference():
    import alea_b200
    ref = golden("chain_heg10.json")
    p = ref["params"]
    setup = golden("setup_heg10.json")
    nw, nw2 = p["nw"], p["dmc_nw"]
    v = alea_b200.Walkers(setup, capacity=nw)
    v.upload(np.array(ref["initial_positions"]))
    v.vmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"])
    rows = v.final_configurations()
    assert np.array_equal(rows.ravel(), np.array(ref["vmc_final_positions"]))
    d = alea_b200.Walkers(setup, capacity=4 * nw2 + 4)
    d.carry_over(v, nw2)
    assert d.nw == nw2
    pos = d.download()["positions"].reshape(nw2, -1)
    assert np.array_equal(pos, rows.reshape(nw, -1)[np.arange(nw2) % nw])
    res, blocks = d.dmc_run(p["dmc_eq"], p["dmc_acc"], p["dmc_steps"], 1, p["dmc_tau"], nw2, p["dmc_seed"],
                            target=nw2)
    want, _ = chain_blocks(ref, p)
    assert np.max(np.abs(np.array(blocks) - want) / np.abs(want)) < 1e-10
    fin = np.array(ref["final_positions"]).reshape(-1, setup["np"] * 2)
    assert d.nw == fin.shape[0]                                    # same branching history
    got = d.final_configurations().reshape(d.nw, -1)
    assert np.max(np.abs(got - fin)) < 1e-9 * np.abs(fin).max()


@pytest.mark.gpu
def test_seed_walker_rows_cycles_and_evaluates():
    import alea_b200
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"])     # 4 walkers
    a = alea_b200.Walkers(setup, capacity=16)
    a.upload(pos)
    ref = a.download()
    b = alea_b200.Walkers(setup, capacity=16)
    b.seed_walker_rows(pos, 10)
    got = b.download()
    idx = np.arange(10) % 4
    assert np.array_equal(got["positions"], ref["positions"][idx])
    assert np.array_equal(got["local_energy"], ref["local_energy"][idx])
    assert np.array_equal(got["weights"], np.ones(10))


@pytest.mark.gpu
def test_carry_over_state_keeps_records():
    import alea_b200
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"])
    a = alea_b200.Walkers(setup, capacity=8)
    a.upload(pos)
    a.set_streams(3, alea_b200.STREAM_VMC, 4)
    for _ in range(5):
        a.vmc_step(225.0, 2)
    src = a.download()
    s = alea_b200.Walkers(setup, capacity=16)
    s.carry_over(a, 6, keep_state=True)
    got = s.download()
    idx = np.arange(6) % 4
    for k in ("positions", "log_psi", "local_energy", "grad", "lap"):
        assert np.array_equal(got[k], src[k][idx]), k
    assert np.array_equal(got["weights"], np.ones(6))
    # the same walkers re-evaluated from their positions agree to rounding
    p = alea_b200.Walkers(setup, capacity=16)
    p.carry_over(a, 6)
    fresh = p.download()
    assert np.array_equal(fresh["positions"], got["positions"])
    assert np.max(np.abs(fresh["local_energy"] - got["local_energy"])) < 1e-10 * np.abs(got["local_energy"]).max()
    # records of another system are refused; its positions are not
    other = dict(setup, pade=[dict(t, b=[0.31]) for t in setup["pade"]])
    o = alea_b200.Walkers(other, capacity=8)
    with pytest.raises(alea_b200.AleaGpuError):
        o.carry_over(a, 4, keep_state=True)
    o.carry_over(a, 4)
    assert o.nw == 4


@pytest.mark.gpu
def test_dmc_milestone_checkpoints_match_reference(tmp_path):
    """alea_gpu_dmc_run's checkpoint hook fires where DMC::run's does (eq,
    a25, a50, a75), with the same population; the hook writes a checkpoint
    file per milestone as the reference's App does (wk.<tag>.*)."""
    import alea_b200
    from alea_b200 import checkpoint as C
    ref = golden("ckpt_dmc_heg10.json")
    p = ref["params"]
    setup = golden("setup_heg10.json")
    nw = p["nw"]
    g = alea_b200.Walkers(setup, capacity=4 * nw + 4)
    g.upload(np.array(ref["initial_positions"]))
    seen = []

    def hook(w, tag, done):
        rows = w.final_configurations()
        seen.append((tag, done, rows))
        C.write_walkers(str(tmp_path / f"wk.{tag}.npz"), rows, lattice=setup["cell"]["vectors"], tag=tag,
                        blocks_done=done)

    g.set_checkpoint_hook(hook)
    g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"], target=nw)
    assert [(t, d) for t, d, _ in seen] == [(c["tag"], c["blocks_done"]) for c in ref["checkpoints"]]
    for (tag, done, rows), c in zip(seen, ref["checkpoints"]):
        want = np.array(c["positions"]).reshape(-1, c["nw"]).T.reshape(c["nw"], -1, 2)
        assert rows.shape == want.shape
        assert np.max(np.abs(rows - want)) < 1e-9 * np.abs(want).max()
        wf = C.read_walkers(str(tmp_path / f"wk.{tag}.npz"))
        assert wf["tag"] == tag and wf["blocks_done"] == done and np.array_equal(wf["positions"], rows)
