"""The reference-side drop-in: GpuVMC / GpuDMC, drivers of the reference's
Driver interface (alea_b200/adapter), on a system the reference's own
components were built for and flattened by pack_system, against the
reference's VMC::run / DMC::run on copies of the same ensemble
(oracle/_ref/ref_harness_gpu, mode gpu_pair).

Tolerances: VMC without drift, final configurations bit for bit and block
energies 1e-10; DMC, block energies 1e-10 (the same branching history),
the same final population, configurations 1e-9.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_harness_gpu")

pytestmark = pytest.mark.gpu

HEG10 = ["system=heg", "nu=5", "nd=5", "rs=30"]


def pair(*args):
    if not os.path.exists(EXE):
        pytest.fail("oracle/_ref/ref_harness_gpu is not built (make -C oracle gpu)")
    out = subprocess.run([EXE, "gpu_pair", *args], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout)


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-12)))


def test_gpu_vmc_driver_equals_reference_vmc():
    r = pair("method=vmc", "nw=6", "seed=11", "eq=1", "acc=2", "steps=3", "substeps=2", "tau=225", *HEG10)
    assert np.array_equal(r["gpu_final_positions"], r["ref_final_positions"])
    assert rel(r["gpu_block_energies"], r["ref_block_energies"]) < 1e-10
    assert r["gpu_acceptance"] == pytest.approx(r["ref_acceptance"], rel=1e-15)


@pytest.mark.parametrize("threads", [8, 2])
def test_gpu_dmc_driver_equals_reference_dmc(threads):
    r = pair("method=dmc", "nw=8", "seed=5", "eq=1", "acc=2", "steps=4", "substeps=2", "tau=2",
             f"threads={threads}", *HEG10)
    assert rel(r["gpu_block_energies"], r["ref_block_energies"]) < 1e-10
    assert r["gpu_energy"] == pytest.approx(r["ref_energy"], rel=1e-10)
    fin_g = np.array(r["gpu_final_positions"])
    fin_r = np.array(r["ref_final_positions"])
    assert fin_g.shape == fin_r.shape
    assert np.max(np.abs(fin_g - fin_r)) < 1e-9 * np.abs(fin_r).max()
    assert r["gpu_method"] == "dmc" and r["gpu_summary"].startswith("dmc: E = ")
