"""Extract the RRTMG-SW coefficient tables from the Fortran DATA statements.

The k-distribution, solar-source and cloud-optics coefficients of RRTMG-SW
are compile-time DATA in ``physics/Radiation/RRTMG/radsw_datatb.f`` (modules
``module_radsw_ref``, ``module_radsw_cldprtb``, ``module_radsw_sflux`` and
``module_radsw_kgb16`` .. ``module_radsw_kgb29``); the band layout is in
``physics/Radiation/RRTMG/radsw_param.f``.  The statement and array-section
parsing is shared with the longwave extractor (``extract_tables.py``); this
file adds the forms that only the shortwave tables use:

* ``integer, parameter :: MFS01 = 1`` inside a table module;
* scalar reals (``real :: a0s, a1s``) filled by ``data a0r,a1r / v, v /``;
* ``real, parameter, public :: rayl = 2.91e-10`` and the one quotient
  ``scalekur = 50.15/48.37``.

Outputs, beside this script:

* ``rrtmg_sw_tables.bin`` -- every array and scalar as little-endian float64
  in the order of the layout header, each array in Fortran (column-major)
  order (integer tables such as ``layreffr`` are stored as exact doubles);
* ``rrtmg_sw_table_layout.h`` -- offsets, shapes and a SHA-256 of the blob.

Literals are parsed as binary64 (promoted-real build, as for the longwave
tables).

Usage (run where the reference tree is readable):
    python extract_sw_tables.py /path/to/ccpp-physics [--out DIR]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import struct
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from extract_tables import _parse_dims, _parse_value, _split_top, _statements, _eval_int  # noqa: E402

# Per-band arrays the SW column path reads (blob name b<NN>_<name>).
_BAND_ARRAYS = ["absa", "absb", "selfref", "forref", "rayl", "rayla", "raylb",
                "absch4", "abso3a", "abso3b", "absco2", "absh2o", "givfac"]
_CLOUD = ["extliq1", "ssaliq1", "asyliq1", "extliq2", "ssaliq2", "asyliq2",
          "extice2", "ssaice2", "asyice2", "extice3", "ssaice3", "asyice3",
          "abari", "bbari", "cbari", "dbari", "ebari", "fbari",
          "a0s", "a1s", "b0s", "b1s", "c0s", "a0r", "a1r", "b0r", "c0r"]
_SFLUX = ["strrat", "specwt", "layreffr", "ix1", "ix2", "ibx",
          "sfluxref01", "sfluxref02", "sfluxref03", "scalekur"]


def _int_params(path, params):
    """Integer parameters: ``integer, parameter :: X = 1`` and
    ``parameter (A=1, B=A+2)`` (sums of names and literals)."""
    def ev(expr):
        tot = 0
        for term in re.split(r"\+", expr):
            term = term.strip()
            if re.fullmatch(r"\d+", term):
                tot += int(term)
            else:
                tot += params[term]
        return tot

    for _, _, st in _statements(path):
        low = st.lower()
        m = re.match(r"integer\s*,\s*parameter\s*(?:,\s*public\s*)?::\s*(\w+)\s*=\s*([\w+\s-]+)$", low)
        if m:
            try:
                params[m.group(1)] = ev(m.group(2))
            except KeyError:
                pass
            continue
        m = re.match(r"parameter\s*\((.*)\)\s*$", low)
        if m:
            for a in _split_top(m.group(1)):
                k, v = a.split("=")
                try:
                    params[k.strip()] = ev(v)
                except KeyError:
                    pass


def _real_expr(expr):
    """A real literal or a quotient of two literals, in binary64."""
    parts = expr.split("/")
    vals = [_parse_value(p, False)[0] for p in parts]
    v = vals[0]
    for d in vals[1:]:
        v = v / d
    return v


def extract(ref_root):
    rrtmg = os.path.join(ref_root, "physics/Radiation/RRTMG")
    params: dict = {}
    _int_params(os.path.join(rrtmg, "radsw_param.f"), params)
    datatb = os.path.join(rrtmg, "radsw_datatb.f")
    _int_params(datatb, params)

    decls, values, filled, src = {}, {}, {}, {}

    def declare(module, name, dims, ln):
        decls[(module, name)] = dims
        size = int(np.prod([hi - lo + 1 for lo, hi in dims])) if dims else 1
        values[(module, name)] = np.full(size, np.nan)
        filled[(module, name)] = np.zeros(size, dtype=bool)
        src[(module, name)] = ln

    for ln, module, st in _statements(datatb):
        if not module:
            continue
        low = st.lower()
        m = re.match(r"real\s*\(\s*kind\s*=\s*kind_phys\s*\)\s*,\s*parameter\s*(?:,\s*public\s*)?::\s*"
                     r"(\w+)\s*=\s*([-+.\deE/]+)\s*$", low)
        if m:
            declare(module, m.group(1), [], ln)
            values[(module, m.group(1))][0] = _real_expr(m.group(2))
            filled[(module, m.group(1))][0] = True
            continue
        m = re.match(r"(real|integer)\b(.*?)::(.*)$", low)
        if m:
            attrs, names = m.group(2), m.group(3)
            if "parameter" in attrs:
                continue
            dm = re.search(r"dimension\s*\(([^)]*)\)", attrs)
            common = _parse_dims(dm.group(1), params) if dm else []
            for item in _split_top(names):
                item = item.strip()
                if not item:
                    continue
                im = re.match(r"(\w+)\s*(?:\((.*)\))?\s*$", item)
                name = im.group(1)
                if name.startswith(("ms", "mf")) and not im.group(2) and not dm and m.group(1) == "integer":
                    continue            # size parameters declared before their parameter statement
                dims = _parse_dims(im.group(2), params) if im.group(2) else common
                declare(module, name, dims, ln)
            continue
        m = re.match(r"data\s+(.*)$", st, flags=re.I | re.S)
        if not m:
            continue
        body = m.group(1)
        # groups "targets / values /" where targets is a comma list of names
        # (scalars) or one array section
        for tm in re.finditer(r"((?:[A-Za-z_]\w*\s*(?:\([^/]*\))?\s*,\s*)*[A-Za-z_]\w*\s*(?:\([^/]*\))?)\s*/([^/]*)/",
                              body):
            targets = _split_top(tm.group(1))
            vals = []
            for tok in tm.group(2).split(","):
                if tok.strip():
                    vals.extend(_parse_value(tok, False))
            pos = 0
            for tgt in targets:
                tgt = tgt.strip()
                nm = re.match(r"([A-Za-z_]\w*)\s*(\(.*\))?$", tgt)
                key = (module, nm.group(1).lower())
                dims = decls[key]
                sub = nm.group(2)
                if not dims:
                    lin = np.zeros(1, dtype=np.int64)
                else:
                    if sub:
                        ranges = []
                        for s, (lo, hi) in zip(_split_top(sub.strip()[1:-1]), dims):
                            s = s.strip()
                            if s == ":":
                                ranges.append(range(lo, hi + 1))
                            elif ":" in s:
                                a, b = s.split(":")
                                ranges.append(range(_eval_int(a, params), _eval_int(b, params) + 1))
                            else:
                                v = _eval_int(s, params)
                                ranges.append(range(v, v + 1))
                    else:
                        ranges = [range(lo, hi + 1) for lo, hi in dims]
                    grids = np.meshgrid(*[np.array(list(r), dtype=np.int64) for r in ranges], indexing="ij")
                    lin = np.zeros(grids[0].shape, dtype=np.int64)
                    stride = 1
                    for g, (lo, hi) in zip(grids, dims):
                        lin += (g - lo) * stride
                        stride *= hi - lo + 1
                    lin = lin.reshape(-1, order="F")
                take = vals[pos:pos + lin.size]
                if len(take) != lin.size:
                    raise ValueError(f"{datatb}:{ln}: {key[1]} expects {lin.size} values, got {len(take)}")
                if filled[key][lin].any():
                    raise ValueError(f"{datatb}:{ln}: {key[1]} element assigned twice")
                values[key][lin] = take
                filled[key][lin] = True
                pos += lin.size
            if pos != len(vals):
                raise ValueError(f"{datatb}:{ln}: {len(vals) - pos} values left over")
    return params, decls, values, filled, src


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("ref_root")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args(argv)
    params, decls, values, filled, src = extract(a.ref_root)

    entries = []

    def add(module, name, cname):
        key = (module, name)
        if key not in values:
            return
        if not filled[key].all():
            raise ValueError(f"{module}:{name} has {int((~filled[key]).sum())} unassigned elements")
        ext = [hi - lo + 1 for lo, hi in decls[key]]
        entries.append((cname, name, ext, values[key], src[key]))

    for nm in ("preflog", "tref"):
        add("module_radsw_ref", nm, nm)
    for nm in _CLOUD:
        add("module_radsw_cldprtb", nm, nm)
    for nm in _SFLUX:
        add("module_radsw_sflux", nm, nm)
    for b in range(16, 30):
        for nm in _BAND_ARRAYS:
            add(f"module_radsw_kgb{b}", nm, f"b{b}_{nm}")

    off = 0
    blob = bytearray()
    lines = []
    for cname, name, ext, vals, ln in entries:
        pad = (-off) % 8
        blob += struct.pack(f"<{pad}d", *([0.0] * pad))
        off += pad
        lines.append((cname, name, off, ext, ln))
        blob += struct.pack(f"<{vals.size}d", *vals.tolist())
        off += vals.size
    sha = hashlib.sha256(bytes(blob)).hexdigest()
    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, "rrtmg_sw_tables.bin"), "wb") as fh:
        fh.write(bytes(blob))
    hdr = [
        "/* Generated by extract_sw_tables.py from radsw_datatb.f (module_radsw_ref,",
        " * module_radsw_cldprtb, module_radsw_sflux, module_radsw_kgb16..29).",
        " * Offsets are in doubles into rrtmg_sw_tables.bin; arrays are stored in",
        " * Fortran order (first index fastest); scalars take one double. Do not edit. */",
        "#pragma once",
        f"#define RRTMG_SW_TABLES_NDOUBLE {off}",
        f"#define RRTMG_SW_TABLES_SHA256 \"{sha}\"",
        "namespace swtab {",
    ]
    for cname, name, o, ext, ln in lines:
        hdr.append(f"constexpr int {cname} = {o};  /* {name}{tuple(ext)} radsw_datatb.f:{ln} */")
    hdr.append("}  // namespace swtab")
    hdr.append("")
    with open(os.path.join(a.out, "rrtmg_sw_table_layout.h"), "w") as fh:
        fh.write("\n".join(hdr))
    manifest = {"sha256": sha, "ndouble": off,
                "arrays": {c: {"name": n, "offset": o, "shape": e, "line": ln} for c, n, o, e, ln in lines}}
    with open(os.path.join(a.out, "rrtmg_sw_tables.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print(f"wrote {len(lines)} arrays, {off} doubles, sha256 {sha}")


if __name__ == "__main__":
    sys.exit(main())
