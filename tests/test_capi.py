"""The C-ABI library builds, loads and exports every symbol include/alea_gpu.h
declares; host-side validation errors come back as status codes (CPU only)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def header_functions():
    text = open(os.path.join(ROOT, "include", "alea_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(alea_gpu_\w+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    names = header_functions()
    for n in ["alea_gpu_create", "alea_gpu_destroy", "alea_gpu_upload_walkers", "alea_gpu_move",
              "alea_gpu_vmc_step", "alea_gpu_dmc_advance", "alea_gpu_dmc_branch",
              "alea_gpu_vmc_run", "alea_gpu_dmc_run"]:
        assert n in names


def test_library_loads_and_exports_every_symbol():
    from alea_b200 import _capi
    lib = _capi.load()
    for name in header_functions():
        assert hasattr(lib, name), name
    assert set(_capi.EXPORTS) >= set(header_functions())
    assert lib.alea_gpu_abi_version() == 1


def test_struct_layout_matches_header():
    """Compile a probe against the header and compare sizes/offsets with ctypes."""
    import subprocess
    import tempfile
    from alea_b200 import _capi
    src = r"""
#include <stddef.h>
#include <stdio.h>
#include "alea_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(alea_gpu_system),
         sizeof(alea_gpu_pair_term), sizeof(alea_gpu_orbitals), sizeof(alea_gpu_ewald),
         offsetof(alea_gpu_system, terms), offsetof(alea_gpu_system, ewald),
         offsetof(alea_gpu_system, coulomb), sizeof(alea_gpu_run_config),
         sizeof(alea_gpu_step_stats), sizeof(alea_gpu_run_result),
         offsetof(alea_gpu_run_result, n_moves), sizeof(alea_gpu_job), offsetof(alea_gpu_job, run),
         sizeof(alea_gpu_job_result), offsetof(alea_gpu_job_result, footprint_bytes));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    want = [ctypes.sizeof(_capi.System), ctypes.sizeof(_capi.PairTerm), ctypes.sizeof(_capi.Orbitals),
            ctypes.sizeof(_capi.Ewald), _capi.System.terms.offset, _capi.System.ewald.offset,
            _capi.System.coulomb.offset, ctypes.sizeof(_capi.RunConfig),
            ctypes.sizeof(_capi.StepStats), ctypes.sizeof(_capi.RunResult),
            _capi.RunResult.n_moves.offset, ctypes.sizeof(_capi.Job), _capi.Job.run.offset,
            ctypes.sizeof(_capi.JobResult), _capi.JobResult.footprint_bytes.offset]
    assert got == want


def test_create_reports_errors_without_crashing():
    from alea_b200 import _capi
    lib = _capi.load()
    ctx = ctypes.c_void_p()
    rc = lib.alea_gpu_create(None, 0, 4, ctypes.byref(ctx))
    assert rc != 0
    assert lib.alea_gpu_last_error(None)
    assert not ctx.value
