"""Oracle package: the CPU checker for the B200 walker hot path.

TEST INFRASTRUCTURE ONLY.  Importable by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg, never by the product package.

* ``liboracle.so`` (built from ``alea_oracle.c``) is a plain-C restatement of
  the reference's VMC/DMC walker algorithms.
* ``_ref/ref_harness`` (built by ``make -C oracle ref`` from the reference's
  own sources, when the reference tree is present) runs the reference itself;
  it pins the restatement and provides the timed CPU baseline.
"""
from .oracle import (  # noqa: F401
    Oracle,
    blob_from_setup,
    ref_harness_path,
    run_ref_harness,
    load_oracle_lib,
)
