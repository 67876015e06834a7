"""The FP32 form of the sweeps (alea_gpu_set_precision) against FP64 on the
same walkers: after FP32 VMC and DMC steps, the local energies the FP32 path
reports agree with an FP64 re-evaluation of the same positions to 1e-5 Ha
per particle, and ln|psi| to 1e-4 per particle (FP32 ratios accumulated in
FP64).  Systems the FP32 form does not take are refused."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,tau,dtau", [("heg42", 225.0, 0.5), ("heg10", 225.0, 0.5)])
def test_fp32_sweeps_match_an_fp64_evaluation(name, tau, dtau):
    import alea_b200
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    pos = np.concatenate([pos] * 16)
    nw, npart = pos.shape[0], setup["np"]
    g = alea_b200.Walkers(setup, capacity=4 * nw + 4)
    g.upload(pos)
    g.set_precision("fp32")
    g.set_streams(5, alea_b200.STREAM_VMC, nw)
    for _ in range(3):
        st = g.vmc_step(tau, 2, False)
        assert 0.05 < st.n_accepted / st.n_proposed < 0.99
    g.vmc_step(dtau, 1, True)
    g.set_streams(5, alea_b200.STREAM_DMC, nw)
    e0 = float(np.mean(g.download()["local_energy"]))
    for _ in range(3):
        g.dmc_advance(dtau, 1, e0, e0, 10.0, 15.0)
    d32 = g.download()
    g.set_precision("fp64")              # re-evaluates the same walkers in FP64
    d64 = g.download()
    assert np.array_equal(d32["positions"], d64["positions"])
    assert np.max(np.abs(d32["local_energy"] - d64["local_energy"])) < 1e-5 * npart
    assert np.max(np.abs(d32["log_psi"] - d64["log_psi"])) < 1e-4 * npart
    g.close()


def test_fp32_refuses_other_systems():
    import alea_b200
    for name in ["heg10t", "dipoles16", "crystal16"]:
        g = alea_b200.Walkers(golden(f"setup_{name}.json"), capacity=4)
        with pytest.raises(alea_b200.AleaGpuError):
            g.set_precision("fp32")
        g.close()
