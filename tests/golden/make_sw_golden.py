"""Generate the shortwave golden fixtures under tests/golden/.

oracle_sw_*.npz -- fluxes, heating rates and surface components of the CPU
restatement of rrtmg_sw_run (oracle/rrtmg_sw_oracle.cpp) for small slices of
the synthetic shortwave workload: regression pins for the restatement and
reference values for the GPU parity tests.  The restatement itself is
unpinned by the reference (no Fortran compiler, no reference tests for this
path); its pieces are checked in tests/test_sw_cpu.py.

Run from the repository root:
    python tests/golden/make_sw_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

# slices of the shortwave leg's workload (16,384 x 127, McICA max-random)
# and of its decorrelation-length and grid-mean variants
CASES = {
    "sw_allsky_127lay": dict(npts=24, nlay=127, seed=41, flags=dict(iovr=1, isubcsw=2)),
    "sw_dcorr_127lay": dict(npts=16, nlay=127, seed=42, flags=dict(iovr=3, isubcsw=2)),
    "sw_gridmean_64lay": dict(npts=16, nlay=64, seed=43, flags=dict(iovr=1, isubcsw=0)),
}


def profile(case):
    from ccpp_physics_b200 import rrtmg_sw as sw, synthetic
    prof = synthetic.make_profiles(case["npts"], case["nlay"], seed=case["seed"])
    return sw.add_sw_inputs(prof, seed=case["seed"], night_fraction=0.2, precip=True)


def main():
    from ccpp_physics_b200 import rrtmg_sw as sw
    from oracle import oracle_sw
    rc, msg = oracle_sw.rswinit()
    assert rc == 0, msg
    for name, case in CASES.items():
        prof = profile(case)
        out = sw.alloc_outputs(case["npts"], case["nlay"], hswb=True, flxprf=True)
        rc, msg = oracle_sw.run(prof, out, flags=case["flags"])
        assert rc == 0, msg
        np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
