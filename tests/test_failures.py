"""Failure detection without a GPU fault: bad inputs come back as status
codes and the context stays usable (the reference throws at the same points:
a singular determinant at evaluation, src/wavefunction/slater_determinant.cpp:
927-928).  Nonfinite positions are refused on the host before any launch;
coincident same-spin electrons give a finite configuration whose determinant
is singular, which the device evaluation flags per walker."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def test_nonfinite_positions_are_refused_on_the_host():
    import alea_b200
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"]).reshape(4, 10, 2)
    g = alea_b200.Walkers(setup, capacity=8)
    bad = pos.copy()
    bad[2, 3, 1] = np.nan
    with pytest.raises(alea_b200.AleaGpuError) as e:
        g.upload(bad)
    assert e.value.code == 1
    with pytest.raises(alea_b200.AleaGpuError):
        g.seed_walker_rows(bad, 4)
    g.upload(pos)                          # still usable
    assert np.all(np.isfinite(g.download()["local_energy"]))


def test_singular_determinant_is_reported_and_the_context_recovers():
    import alea_b200
    setup = golden("setup_heg10.json")
    pos = np.array(golden("eval_heg10.json")["positions"]).reshape(4, 10, 2)
    g = alea_b200.Walkers(setup, capacity=8)
    bad = pos.copy()
    bad[1, 1] = bad[1, 0]                  # two up electrons on one point: equal rows of D
    with pytest.raises(alea_b200.AleaGpuError) as e:
        g.upload(bad)
    assert e.value.code == 4 and "walker 1" in str(e.value)
    g.upload(pos)
    g.set_streams(1, alea_b200.STREAM_VMC, 4)
    st = g.vmc_step(225.0, 1)
    assert st.n_walkers == 4 and np.isfinite(st.energy_sum)
