"""Regenerate the golden fixtures in this directory from the compiled reference.

    make -C oracle ref            # builds oracle/_ref/ref_harness from the reference tree
    python tests/golden/make_fixtures.py

Every fixture is the output of the reference's own code (its VMC/DMC drivers,
components and setup-time breakups) run through oracle/_ref/ref_harness:

* ``setup_<name>.json``  system description: cell, groups, orbitals, Padé /
  Drummond parameters, image-sum and Ewald tables (the reference's breakups);
* ``eval_<name>.json``   4 walkers from the reference App's initialisation
  (mt19937_64, seed 12345): ln|psi|, E_L, gradients, Laplacians;
* ``vmc_<name>.json``    VMC::run with one stream per walker (threads = nw):
  initial positions, per-walker E_L of every accumulation step, final
  positions, acceptance;
* ``dmc_<name>.json``    DMC::run with one crowd per walker: per-step
  populations, weights, energies, ids, final positions;
* ``est_<name>.json``     the estimators (PairCorrelation, Density,
  StructureFactor) accumulated over fixed configurations (fresh App
  initialisations) with given weights: configurations, weights, series;
* ``est_vmc_<name>.json`` / ``est_dmc_<name>.json`` the same estimators
  attached to VMC::run / DMC::run (runs as in vmc_/dmc_<name>): series;
* ``fw_dmc_<name>.json``  a DMC::run with forward walking (pure potential energy
  and pure estimators at three lags): the run result's series and scalars;
* ``ckpt_dmc_<name>.json`` a DMC::run's milestone checkpoint calls (eq, a25,
  a50, a75): tag, blocks done, the population's positions;
* ``chain_<name>.json``   a VMC::run whose final configurations seed a DMC::run
  (carry_over_walkers): DMC populations and weighted energy sums per step;
* ``dmcstat_<name>.json`` a long DMC::run on 8 crowds: per-step Σw and ΣwE_L,
  reduced here to accumulation-block energies, their mean and its reblocked
  standard error (the statistical reference for the device's DMC);
* ``vmcstat_<name>.json`` a VMC::run of the VMC benchmark's shape (512
  walkers, 8 threads): block energies, their reblocked mean and error;
* ``vmc_<name>_crowd.json`` / ``dmc_<name>_crowd.json`` VMC::run / DMC::run
  with fewer threads than walkers: each thread's stream serves a contiguous
  range of walkers (VMC's per-thread clones, DMC's crowds).
"""
from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import run_ref_harness  # noqa: E402

SYSTEMS = {
    "exciton": dict(system="exciton"),
    "heg10": dict(system="heg", nu=5, nd=5, rs=30),
    "crystal16": dict(system="crystal", nx=4, ny=4, rs=40),
    "heg42": dict(system="heg", nu=21, nd=21, rs=30),
    "dipoles16": dict(system="dipoles", n=16),
    "heg10t": dict(system="heg", nu=5, nd=5, rs=30, tx=0.25, ty=0.125),
    "heg10bf": dict(system="heg", nu=5, nd=5, rs=30, bf=1),
    # the 10 x 12 Wigner crystal (120 electrons, 60 per spin) at r_s = 40
    "crystal120": dict(system="crystal", nx=10, ny=12, rs=40),
    # the crystal with its Drummond alpha_0, an alpha_2 term and L optimisable
    "crystal16p": dict(system="crystal", nx=4, ny=4, rs=40, drummond_free=1, alpha0=-2e-3,
                       alpha2=3e-8, gauss_free=1),
    # 3-D electron gases (the reference's backflow determinant, Drummond
    # Jastrow and kinetic energy in a cubic cell, plane waves passed
    # directly): the 54-electron backflow gas at r_s = 5, a 14-electron one,
    # and the 54-electron plain plane-wave determinant without a Jastrow
    "heg54bf3d": dict(system="heg3d", nu=27, nd=27, rs=5, alpha0=-0.01),
    "heg14bf3d": dict(system="heg3d", nu=7, nd=7, rs=5, alpha0=-0.01, bf_un1=0.02),
    "heg54pw3d": dict(system="heg3d", nu=27, nd=27, rs=5, bf=0, jastrow=0),
    # the same gases with cusp-free Jastrows, for DMC: with the kinetic energy
    # alone a Coulomb cusp leaves an unbalanced 1/r local energy
    "heg14bf3ds": dict(system="heg3d", nu=7, nd=7, rs=5, alpha0=-0.01, bf_un1=0.02, cusp=0),
    "heg54bf3ds": dict(system="heg3d", nu=27, nd=27, rs=5, alpha0=-0.01, cusp=0),
    # open 3-D cell, the reference's own 3-D backflow test shape: Gaussian
    # orbitals, two backflow channels, a Padé Jastrow and open Coulomb
    "gauss3d": dict(system="gauss3d"),
    # the 14-electron gas with its backflow determinant alone, for the
    # statistical DMC comparison (kinetic energy only: stable weights)
    "heg14bf3dp": dict(system="heg3d", nu=7, nd=7, rs=5, jastrow=0),
}
VMC = {
    "exciton": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=0.05),
    "heg10": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=225.0),
    "heg10_drift": dict(nw=6, seed=13, eq=1, acc=2, steps=3, substeps=1, tau=225.0, drift=1),
    "crystal16": dict(nw=4, seed=17, eq=0, acc=2, steps=2, substeps=1, tau=400.0),
    "dipoles16": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=0.0003),
    "heg10t": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=225.0),
    "heg10t_drift": dict(nw=6, seed=13, eq=1, acc=2, steps=3, substeps=1, tau=225.0, drift=1),
    "heg10bf": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=225.0),
    "heg10bf_drift": dict(nw=6, seed=13, eq=1, acc=2, steps=3, substeps=1, tau=225.0, drift=1),
    "crystal120": dict(nw=4, seed=19, eq=0, acc=1, steps=2, substeps=1, tau=400.0),
    "heg54bf3d": dict(nw=4, seed=11, eq=0, acc=1, steps=2, substeps=1, tau=4.0),
    "heg14bf3d": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=4.0),
    "heg14bf3d_drift": dict(nw=6, seed=13, eq=1, acc=2, steps=3, substeps=1, tau=1.0, drift=1),
    "heg54pw3d": dict(nw=4, seed=11, eq=0, acc=1, steps=2, substeps=1, tau=4.0),
    "gauss3d": dict(nw=6, seed=11, eq=1, acc=2, steps=3, substeps=2, tau=0.1),
    "gauss3d_drift": dict(nw=6, seed=13, eq=1, acc=2, steps=3, substeps=1, tau=0.05, drift=1),
}
DMC = {
    "exciton": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=0.05),
    "heg10": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=2.0),
    "dipoles16": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=1e-5),
    "heg10t": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=2.0),
    "heg10bf": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=2.0),
    "heg42": dict(nw=16, seed=5, eq=1, acc=2, steps=3, substeps=1, tau=0.5),
    "heg14bf3ds": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=0.005),
    "heg54bf3ds": dict(nw=8, seed=5, eq=1, acc=1, steps=2, substeps=1, tau=0.005),
    "gauss3d": dict(nw=8, seed=5, eq=1, acc=2, steps=4, substeps=2, tau=0.01),
}

# Fewer threads (streams, crowds) than walkers: contiguous walker ranges.
VMC_CROWD = {"heg42": dict(nw=64, seed=11, eq=1, acc=2, steps=2, substeps=1, tau=225.0, threads=4)}
DMC_CROWD = {"heg42": dict(nw=32, seed=5, eq=1, acc=2, steps=3, substeps=1, tau=0.5, threads=4)}


# Observable estimators (gofr / density / sofk), with the argument names of
# ref_harness's estimator builder.
EST = {
    "heg10": dict(gofr_rmax=80.0, gofr_bins=20, dens_rmax=84.0, dens_bins=8, sofk_kmax=0.12),
    "dipoles16": dict(gofr_rmax=0.13, gofr_bins=13, dens_rmax=0.14, dens_bins=4, dens_pp=1,
                      sofk_kmax=60.0),
    "crystal16": dict(gofr_rmax=130.0, gofr_bins=26, dens_rmax=200.0, dens_bins=10, sofk_kmax=0.05),
}
ESTIMATE = {
    "heg10": dict(nw=6, acc=3, steps=2, init_seed=77),
    "dipoles16": dict(nw=5, acc=2, steps=3, init_seed=78),
}
EST_VMC = {"heg10": "heg10", "dipoles16": "dipoles16", "crystal16": "crystal16"}
EST_DMC = {"heg10": "heg10"}

# Forward walking (pure estimators) on a DMC run: lags in imaginary time.
FW = {"heg10": dict(fw_lags="0,4,8", fw_interval=1)}

# VMC -> DMC stage chain: DMC seeded from VMC's final configurations.
CHAIN = {
    "heg10": dict(nw=6, seed=11, eq=1, acc=1, steps=2, substeps=2, tau=225.0, dmc_nw=8, dmc_eq=1,
                  dmc_acc=2, dmc_steps=3, dmc_tau=2.0, dmc_seed=5),
}

# the VMC benchmark's system and walker count (512 walkers, Metropolis step
# 0.5 rs): block energies for the statistical comparison of the device's VMC
VMC_STAT = {
    "heg42": dict(nw=512, seed=515151, eq=2, acc=24, steps=10, substeps=5, tau=225.0, threads=8),
}

DMC_STAT = {
    "heg10": dict(nw=1024, seed=424242, eq=10, acc=50, steps=10, substeps=1, tau=0.5, threads=8),
    "heg42": dict(nw=1024, seed=424243, eq=10, acc=40, steps=10, substeps=1, tau=0.5, threads=8),
    "heg14bf3dp": dict(nw=1024, seed=424244, eq=10, acc=40, steps=10, substeps=1, tau=0.5, threads=8),
}


def reblock(x):
    """Mean and the largest standard error over pairwise blocking levels with
    at least 8 blocks."""
    import numpy as np
    x = np.asarray(x, dtype=float)
    mean = float(x.mean())
    err = 0.0
    while len(x) >= 8:
        err = max(err, float(x.std(ddof=1) / np.sqrt(len(x))))
        x = 0.5 * (x[0:len(x) // 2 * 2:2] + x[1:len(x) // 2 * 2:2])
    return mean, err


def dump(name, obj):
    with open(os.path.join(HERE, name), "w") as f:
        json.dump(obj, f, separators=(",", ":"))
    print("wrote", name)


CKPT = {"heg10": dict(nw=8, seed=5, eq=1, acc=4, steps=3, substeps=1, tau=2.0, ckpt=1)}


def ckpt_fixtures(only=None):
    for name, run in CKPT.items():
        if only and name not in only:
            continue
        r = run_ref_harness("dmc", **run, **SYSTEMS[name])
        dump(f"ckpt_dmc_{name}.json", {"params": run, "checkpoints": r["checkpoints"],
                                       "initial_positions": r["initial_positions"]})


def fw_fixtures(only=None):
    for name, fw in FW.items():
        if only and name not in only:
            continue
        r = run_ref_harness("dmc", **DMC[name], **EST[name], **fw, **SYSTEMS[name])
        dump(f"fw_dmc_{name}.json", {"params": DMC[name], "est": EST[name], "fw": fw,
                                     "estimators": r["estimators"], "walkers": r["walkers"],
                                     "initial_positions": r["initial_positions"]})


def crowd_fixtures(only=None):
    for name, run in VMC_CROWD.items():
        if only and name not in only:
            continue
        r = run_ref_harness("vmc", **run, **SYSTEMS[name])
        r["params"] = run
        r["system"] = name
        dump(f"vmc_{name}_crowd.json", r)
    for name, run in DMC_CROWD.items():
        if only and name not in only:
            continue
        r = run_ref_harness("dmc", **run, **SYSTEMS[name])
        r["params"] = run
        r["system"] = name
        dump(f"dmc_{name}_crowd.json", r)


def chain_fixtures(only=None):
    for name, run in CHAIN.items():
        if only and name not in only:
            continue
        r = run_ref_harness("chain", **run, **SYSTEMS[name])
        r["params"] = run
        dump(f"chain_{name}.json", r)


# systems that serve only DMC fixtures (no evaluation fixture)
NO_EVAL = {"heg14bf3ds", "heg54bf3ds", "heg14bf3dp"}


def main(only=None):
    for name, args in SYSTEMS.items():
        if only and name not in only:
            continue
        dump(f"setup_{name}.json", run_ref_harness("setup", **args))
        if name in NO_EVAL:
            continue
        ev = run_ref_harness("eval", nw=4, seed=12345, **args)
        ev.pop("mode", None)
        dump(f"eval_{name}.json", ev)
    for name, run in VMC.items():
        sysname = name.split("_")[0]
        if only and sysname not in only:
            continue
        r = run_ref_harness("vmc", **run, **SYSTEMS[sysname])
        r["params"] = run
        r["system"] = sysname
        dump(f"vmc_{name}.json", r)
    for name, run in DMC.items():
        if only and name not in only:
            continue
        r = run_ref_harness("dmc", **run, **SYSTEMS[name])
        r["params"] = run
        r["system"] = name
        dump(f"dmc_{name}.json", r)
    for name, run in ESTIMATE.items():
        if only and name not in only:
            continue
        r = run_ref_harness("estimate", **run, **EST[name], **SYSTEMS[name])
        r["params"] = run
        r["est"] = EST[name]
        dump(f"est_{name}.json", r)
    for name, key in EST_VMC.items():
        if only and name not in only:
            continue
        r = run_ref_harness("vmc", **VMC[key], **EST[name], **SYSTEMS[name])
        dump(f"est_vmc_{name}.json", {"params": VMC[key], "est": EST[name], "estimators": r["estimators"],
                                      "final_positions": r["final_positions"]})
    for name, key in EST_DMC.items():
        if only and name not in only:
            continue
        r = run_ref_harness("dmc", **DMC[key], **EST[name], **SYSTEMS[name])
        dump(f"est_dmc_{name}.json", {"params": DMC[key], "est": EST[name], "estimators": r["estimators"],
                                      "walkers": r["walkers"], "final_positions": r["final_positions"]})
    crowd_fixtures(only)
    chain_fixtures(only)
    fw_fixtures(only)
    ckpt_fixtures(only)
    for name, run in VMC_STAT.items():
        if only and name not in only:
            continue
        r = run_ref_harness("vmc", **run, **SYSTEMS[name])
        mean, err = reblock(r["block_energies"])
        dump(f"vmcstat_{name}.json", {"params": run, "system": name, "block_energies": r["block_energies"],
                                      "energy": mean, "energy_error": err, "acceptance": r["acceptance"]})
    for name, run in DMC_STAT.items():
        if only and name not in only:
            continue
        r = run_ref_harness("bench", method="dmc", **run, **SYSTEMS[name])
        n_acc_steps = run["acc"] * run["steps"]
        w = r["weight_sum"][-n_acc_steps:]
        we = r["weighted_energy_sum"][-n_acc_steps:]
        blocks = [sum(we[b * run["steps"]:(b + 1) * run["steps"]]) /
                  sum(w[b * run["steps"]:(b + 1) * run["steps"]]) for b in range(run["acc"])]
        mean, err = reblock(blocks)
        dump(f"dmcstat_{name}.json", {"params": run, "system": name, "block_energies": blocks,
                                      "energy": mean, "energy_error": err})


if __name__ == "__main__":
    main(set(sys.argv[1:]) or None)   # optional system names: regenerate only those
