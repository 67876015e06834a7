"""The C-ABI library builds, loads and exports every symbol include/alea_gpu.h
declares; host-side validation errors come back as status codes (CPU only)."""
import ctypes
import subprocess
import tempfile
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
    assert lib.alea_gpu_abi_version() == 2


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


def test_every_struct_field_matches_the_header():
    """Every ctypes mirror of an alea_gpu.h struct has the C size and, field by
    field, the C offset (a probe compiled with gcc against the header)."""
    from alea_b200 import _capi
    pairs = [("alea_gpu_spline", _capi.Spline), ("alea_gpu_kset", _capi.KSet), ("alea_gpu_group", _capi.Group),
             ("alea_gpu_orbitals", _capi.Orbitals), ("alea_gpu_pair_term", _capi.PairTerm),
             ("alea_gpu_ewald", _capi.Ewald), ("alea_gpu_coulomb", _capi.Coulomb),
             ("alea_gpu_inverse_power", _capi.InversePower),
             ("alea_gpu_backflow_channel", _capi.BackflowChannel), ("alea_gpu_backflow", _capi.Backflow),
             ("alea_gpu_system", _capi.System), ("alea_gpu_vmc_params", _capi.VmcParams),
             ("alea_gpu_step_stats", _capi.StepStats), ("alea_gpu_dmc_params", _capi.DmcParams),
             ("alea_gpu_run_config", _capi.RunConfig), ("alea_gpu_run_result", _capi.RunResult),
             ("alea_gpu_job", _capi.Job), ("alea_gpu_job_result", _capi.JobResult),
             ("alea_gpu_estimator_spec", _capi.EstimatorSpec), ("alea_gpu_estimator_desc", _capi.EstimatorDesc),
             ("alea_gpu_fw_summary", _capi.FwSummary)]
    lines, want = [], []
    for cname, cls in pairs:
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        want.append(ctypes.sizeof(cls))
        for f in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {f[0]}));')
            want.append(getattr(cls, f[0]).offset)
    src = "#include <stddef.h>\n#include <stdio.h>\n#include \"alea_gpu.h\"\nint main(void) {\n" + \
          "\n".join(lines) + "\n  return 0;\n}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    assert got == want
