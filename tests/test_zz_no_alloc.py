"""alea_gpu_vmc_step_noalloc against alea_gpu_vmc_step.

The allocation-free step keeps its random numbers and statistics in a static
device array shared by every context on the device.  Two contexts on the same
walkers and streams, one stepped through each entry point, must stay equal
over two calls in a row (the second call reuses the array's last contents):
positions and accept counts bit for bit, local energies to the path's 1e-10
relative tolerance, energy sums to 1e-12 relative (reduced on the device in
another order).  The file sorts last so that it also runs after every other
GPU test has used the device.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

E_L_RTOL = 1e-10
SUM_RTOL = 1e-12


def _pair(name="heg10", precision="fp64"):
    import alea_b200
    setup = golden(f"setup_{name}.json")
    pos = np.array(golden(f"eval_{name}.json")["positions"])
    nw = pos.shape[0]
    a = alea_b200.Walkers(setup, capacity=nw)
    b = alea_b200.Walkers(setup, capacity=nw)
    for g in (a, b):
        g.upload(pos)
        if precision != "fp64":
            g.set_precision(precision)
        g.set_streams(5, alea_b200.STREAM_VMC, nw)
    return a, b


# the one-warp FP64 sweep, its FP32 form, and the generic CTA sweep (the
# backflow determinant), each stepped through both entry points
@pytest.mark.parametrize("name,precision", [("heg10", "fp64"), ("heg10", "fp32"), ("heg10bf", "fp64")])
def test_noalloc_step_matches_vmc_step_twice(name, precision):
    a, b = _pair(name, precision)
    for call, (tau, n_sub, drift) in enumerate([(225.0, 2, False), (100.0, 1, True)]):
        sa = a.vmc_step(tau, n_sub, drift)
        sb = b.vmc_step_noalloc(tau, n_sub, drift)
        da, db = a.download(), b.download()
        np.testing.assert_array_equal(db["positions"], da["positions"], err_msg=f"call {call}")
        np.testing.assert_allclose(db["local_energy"], da["local_energy"], rtol=E_L_RTOL)
        assert sb.n_accepted == sa.n_accepted
        assert sb.n_proposed == sa.n_proposed and sb.n_walkers == sa.n_walkers
        assert sb.energy_sum == pytest.approx(sa.energy_sum, rel=SUM_RTOL)
        assert sb.energy_sq_sum == pytest.approx(sa.energy_sq_sum, rel=SUM_RTOL)
        assert b.last_kernel_ms() > 0.0      # the sweep of this call was timed
    a.close()
    b.close()


def test_noalloc_step_rejects_oversized_scratch():
    import alea_b200
    a, b = _pair()
    nw, np_ = b.nw, b.np
    limit = 1048576          # ALEA_GPU_NOALLOC_RANDOMS in include/alea_gpu.h
    n_sub = limit // (np_ * 3 * nw) + 1
    before = b.download()["positions"]
    with pytest.raises(alea_b200.AleaGpuError, match="static scratch"):
        b.vmc_step_noalloc(225.0, n_sub, False)
    # nothing ran, and the context still steps
    np.testing.assert_array_equal(b.download()["positions"], before)
    sa = a.vmc_step(225.0, 1, False)
    sb = b.vmc_step_noalloc(225.0, 1, False)
    np.testing.assert_array_equal(b.download()["positions"], a.download()["positions"])
    assert sb.n_accepted == sa.n_accepted
    a.close()
    b.close()
