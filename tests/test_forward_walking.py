"""Forward walking (pure estimators) of a DMC run, against the compiled
reference's ForwardWalking (src/qmc/forward_walking.cpp) on the same DMC run.

The device's population history equals the reference's (same branching), so
the ancestries, the descendant weights and the kept ancestors are the same;
positions and weights agree to rounding.  Checked: per-block pure potential
energies (1e-9), measurement counts (exact), surviving fractions (1e-12) and
the pure g(r), density and S(k) series (1e-9); lag 0 repeats the mixed
estimate.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_forward_walking_matches_reference():
    import alea_b200
    from test_estimators import compare
    ref = golden("fw_dmc_heg10.json")
    p, est = ref["params"], ref["est"]
    e = ref["estimators"]
    setup = golden("setup_heg10.json")
    nw = p["nw"]
    lags = [float(x) for x in ref["fw"]["fw_lags"].split(",")]
    g = alea_b200.Walkers(setup, capacity=4 * nw + 4)
    g.upload(np.array(ref["initial_positions"]))
    g.set_forward_walking(lags, ref["fw"]["fw_interval"])
    ids = {}
    for i in range(len(lags)):
        ids[i] = [g.add_fw_estimator(i, "gofr", n_bins=est["gofr_bins"], rmax=est["gofr_rmax"]),
                  g.add_fw_estimator(i, "density", n_bins=est["dens_bins"], rmax=est["dens_rmax"]),
                  g.add_fw_estimator(i, "sofk", kmax=est["sofk_kmax"])]
    mixed = g.add_estimator("gofr", n_bins=est["gofr_bins"], rmax=est["gofr_rmax"])
    g.dmc_run(p["eq"], p["acc"], p["steps"], p["substeps"], p["tau"], nw, p["seed"], target=nw)
    for i in range(len(lags)):
        r = g.fw_result(i)
        tag = f"fw{i}"
        assert r["lag_steps"] == int(e[f"{tag}_lag_steps"])
        assert r["measurements"] == int(e[f"{tag}_measurements"])
        assert abs(r["surviving_fraction"] - e[f"{tag}_surviving_fraction"]) < 1e-12
        want = np.array(e[f"acc_block_potential_{tag}"])
        assert r["block_potentials"].shape == want.shape
        assert np.max(np.abs(r["block_potentials"] - want) / np.abs(want)) < 1e-9
        assert abs(r["potential"] - e[f"potential_{tag}"]) < 1e-9 * abs(e[f"potential_{tag}"])
        out = {}
        for k in ids[i]:
            out.update(g.fw_estimator_results(i, k))
        ref_tag = {k: v for k, v in e.items() if f"_{tag}_" in k or k.endswith(f"_{tag}")}
        # S(k) k-vectors are matched by value inside compare()
        ref_tag["sofk_kx"], ref_tag["sofk_ky"] = e[f"sofk_{tag}_kx"], e[f"sofk_{tag}_ky"]
        out["sofk_kx"], out["sofk_ky"] = out[f"sofk_{tag}_kx"], out[f"sofk_{tag}_ky"]
        compare(out, ref_tag, 1e-9, skip=("sofk_kx", "sofk_ky"))
    # lag 0 with every walker kept is the mixed measurement itself
    m = g.estimator_results(mixed)
    f0 = g.fw_estimator_results(0, ids[0][0])
    assert np.allclose(f0["gofr_fw0_up_down"], m["gofr_up_down"], rtol=1e-12, atol=0)


def test_forward_walking_schedule_errors():
    import alea_b200
    setup = golden("setup_heg10.json")
    g = alea_b200.Walkers(setup, capacity=40)
    g.upload(np.array(golden("eval_heg10.json")["positions"]))
    with pytest.raises(alea_b200.AleaGpuError):
        g.set_forward_walking([4.0, 2.0])                   # not increasing
    g.set_forward_walking([0.0, 3.0])                       # 3 is not a whole number of 2.0-steps
    with pytest.raises(alea_b200.AleaGpuError):
        g.dmc_run(1, 1, 4, 1, 2.0, 4, 5, target=4)
    g.set_forward_walking([0.0, 16.0])                      # beyond the 4-step equilibration
    with pytest.raises(alea_b200.AleaGpuError):
        g.dmc_run(1, 1, 4, 1, 2.0, 4, 5, target=4)
    g.set_forward_walking([0.0, 2.0], interval=3)           # does not divide 4 steps per block
    with pytest.raises(alea_b200.AleaGpuError):
        g.dmc_run(1, 1, 4, 1, 2.0, 4, 5, target=4)
    g.set_forward_walking([])
    g.dmc_run(1, 1, 4, 1, 2.0, 4, 5, target=4)
