"""Generate the committed golden fixtures under tests/golden/.

* dtb_literals.json -- spot literals read straight from the DATA text of
  physics/Radiation/RRTMG/radlw_datatb.f (first and last value of the first
  DATA statement of every coefficient array, with its Fortran element
  index), parsed here independently of the table extractor; the tests check
  the shipped table blob against them.
* mt_words.json -- the first raw words and reals of the GFS Mersenne twister
  (random_setseed_t + random_number_t, mersenne_twister.f:285-372) for a
  set of seeds, from the CPU restatement after it was checked against
  numpy's MT19937.
* oracle_*.npz -- fluxes and heating rates of the CPU restatement for small
  slices of the synthetic workloads (regression pins for the restatement
  and the reference values of the GPU parity tests).

Run from the repository root where the reference tree is readable:
    python tests/golden/make_golden.py /path/to/ccpp-physics
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

# small slices of the benchmark configurations used for pinned outputs
CASES = {
    "c1_clear_64lay": dict(npts=24, nlay=64, seed=11, cloudy=False),
    "c2_allsky_127lay": dict(npts=24, nlay=127, seed=12, cloudy=True),
}


def dtb_literals(ref_root):
    path = os.path.join(ref_root, "physics/Radiation/RRTMG/radlw_datatb.f")
    lines = open(path, encoding="ascii", errors="replace").read().split("\n")
    out = []
    seen = set()
    module = None
    i = 0
    while i < len(lines):
        s = lines[i].split("!")[0]
        m = re.match(r"\s*module\s+(module_radlw_\w+)", s, re.I)
        if m:
            module = m.group(1).lower()
        m = re.match(r"\s*data\s+(\w+)\s*(\(([^)]*)\))?\s*/(.*)$", s, re.I)
        if m and module:
            name = m.group(1).lower()
            start = i + 1
            body = m.group(4)
            while "/" not in body:
                i += 1
                body += " " + lines[i].split("!")[0].strip().lstrip("&").rstrip("&")
            body = body.split("/")[0].replace("&", " ")
            toks = [t.strip() for t in body.split(",") if t.strip()]
            key = (module, name)
            if key not in seen:
                seen.add(key)
                sub = m.group(3)
                out.append(dict(module=module, name=name, section=sub, line=start,
                                first=toks[0], last=toks[-1], count=len(toks)))
        i += 1
    return out


def main(argv):
    if len(argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <ccpp-physics source tree>  "
                 "(the checkout whose radlw_datatb.f the DTB literals are read from)")
    ref_root = argv[1]
    lits = dtb_literals(ref_root)
    with open(os.path.join(HERE, "dtb_literals.json"), "w") as fh:
        json.dump(lits, fh, indent=1)

    from oracle import oracle
    from ccpp_physics_b200 import synthetic
    rc, msg = oracle.rlwinit()
    assert rc == 0, msg
    mt = {}
    for seed in (0, 1, 141, 2**31 - 1, -5, 884735):
        u, x, _ = oracle.mt_stream(seed, 1300)
        mt[str(seed)] = dict(u32=[int(v) for v in u[:8]] + [int(u[623]), int(u[624]), int(u[1299])],
                             real=[float(v) for v in x[:8]])
    with open(os.path.join(HERE, "mt_words.json"), "w") as fh:
        json.dump(mt, fh, indent=1)

    for name, cfg in CASES.items():
        prof = synthetic.make_profiles(cfg["npts"], cfg["nlay"], seed=cfg["seed"], cloudy=cfg["cloudy"])
        rc, msg, out = oracle.rrtmg_lw_run(prof, hlw0=True, hlwb=True, flxprf=True)
        assert rc == 0, msg
        np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), **out,
                            cfg=json.dumps(cfg))
    print(f"{len(lits)} DTB literals, {len(mt)} MT seeds, {len(CASES)} oracle cases")


if __name__ == "__main__":
    main(sys.argv)
