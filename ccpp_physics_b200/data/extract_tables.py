"""Extract the RRTMG-LW coefficient tables from the Fortran DATA statements.

The k-distribution, Planck and cloud-optics coefficients of RRTMG-LW are
compile-time DATA in ``physics/Radiation/RRTMG/radlw_datatb.f`` (modules
``module_radlw_avplank``, ``module_radlw_ref``, ``module_radlw_cldprlw`` and
``module_radlw_kgb01`` .. ``module_radlw_kgb16``) and the band layout is in
``physics/Radiation/RRTMG/radlw_param.f:103-142``.  This script parses those
statements (``data name(sub, sub) / v, v, ... /`` with Fortran column-major
array sections and ``&`` continuations) and writes

* ``rrtmg_lw_tables.bin`` -- every array as little-endian float64, packed in
  the order of the layout header, each array in Fortran (column-major) order;
* ``rrtmg_lw_table_layout.h`` -- offsets, shapes and a SHA-256 of the blob.

Values are parsed from the decimal text with ``float()`` (round to nearest
binary64), which is what a Fortran compiler does for promoted-real builds
(``-fdefault-real-8`` / ``-real-size 64``), the precision the ccpp-physics
host builds use for ``kind_phys=8`` physics.  With ``--default-real-4`` the
values are first rounded to binary32 (the un-promoted literal semantics);
that mode exists for studying the literal-precision caveat only.

Usage (run where the reference tree is readable):
    python extract_tables.py /path/to/ccpp-physics [--out DIR]
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

# Arrays that the LW column path reads, in blob order: (module, name).
_BAND_ARRAYS = [
    "absa", "absb", "selfref", "forref", "fracrefa", "fracrefb",
    "ka_mn2", "kb_mn2", "ka_mn2o", "kb_mn2o", "ka_mo3", "kb_mo3",
    "ka_mco2", "kb_mco2", "ka_mo2", "kb_mo2", "ka_mco", "ccl4",
    "cfc11adj", "cfc12", "cfc22adj",
]


def _strip_comment(line: str) -> str:
    i = line.find("!")
    return line if i < 0 else line[:i]


def _statements(path: str):
    """Yield (first_line_number, module, statement_text) for a Fortran file,
    joining ``&`` continuation lines (fixed or free form)."""
    module = None
    cur = None
    cur_line = 0
    with open(path, "r", encoding="ascii", errors="replace") as fh:
        for ln, raw in enumerate(fh, start=1):
            if raw[:1] in ("c", "C", "*") and not raw[:6].strip().lower().startswith(("contains",)):
                # fixed-form comment in column 1 (none of the tables use it)
                if raw[:1] in ("c", "C") and raw[1:2] not in (" ", "\t", "\n", ""):
                    pass
                else:
                    continue
            text = _strip_comment(raw.rstrip("\n"))
            s = text.strip()
            if not s:
                continue
            is_cont = s.startswith("&")
            if is_cont:
                s = s[1:]
            if cur is not None and (is_cont or cur.rstrip().endswith("&")):
                cur = cur.rstrip()
                if cur.endswith("&"):
                    cur = cur[:-1]
                cur += " " + s
                continue
            if cur is not None:
                yield cur_line, module, cur
            low = s.lower()
            m = re.match(r"module\s+(\w+)", low)
            if m and not low.startswith("module procedure"):
                module = m.group(1)
            if re.match(r"end\s+module", low):
                module = None
            cur = s
            cur_line = ln
        if cur is not None:
            yield cur_line, module, cur


def _eval_int(expr: str, params: dict) -> int:
    expr = expr.strip()
    if re.fullmatch(r"[+-]?\d+", expr):
        return int(expr)
    key = expr.lower()
    if key in params:
        return params[key]
    raise KeyError(f"unknown integer parameter {expr!r}")


def _parse_dims(spec: str, params: dict):
    dims = []
    for part in spec.split(","):
        part = part.strip()
        if ":" in part:
            lo, hi = part.split(":")
            dims.append((_eval_int(lo, params), _eval_int(hi, params)))
        else:
            dims.append((1, _eval_int(part, params)))
    return dims


def _split_top(s: str):
    """Split on commas that are not inside parentheses."""
    out, depth, buf = [], 0, []
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(buf))
            buf = []
        else:
            buf.append(ch)
    out.append("".join(buf))
    return out


def _parse_value(tok: str, real4: bool):
    tok = tok.strip().lower().replace("d", "e")
    tok = re.sub(r"_\w+$", "", tok)
    if "*" in tok:
        n, v = tok.split("*")
        return [_parse_value(v, real4)[0]] * int(n)
    v = float(tok)
    if real4 and re.search(r"[.e]", tok):
        v = float(np.float32(v))
    return [v]


def extract(ref_root: str, real4: bool = False):
    param_f = os.path.join(ref_root, "physics/Radiation/RRTMG/radlw_param.f")
    datatb = os.path.join(ref_root, "physics/Radiation/RRTMG/radlw_datatb.f")
    params: dict = {}
    # integer parameters of radlw_param.f (NBANDS, NGPTLW, NG01.., NS01..)
    for _, _, st in _statements(param_f):
        low = st.lower()
        m = re.match(r"integer\s*,\s*parameter\s*::\s*(\w+)\s*=\s*(\d+)", low)
        if m:
            params[m.group(1)] = int(m.group(2))
        m = re.match(r"parameter\s*\((.*)\)\s*$", low)
        if m:
            for a in _split_top(m.group(1)):
                k, v = a.split("=")
                params[k.strip()] = int(v)

    decls: dict = {}      # (module, name) -> dims
    kinds: dict = {}      # (module, name) -> 'real' | 'integer'
    values: dict = {}     # (module, name) -> np.ndarray (flat, Fortran order)
    filled: dict = {}
    real_params: dict = {}
    src_lines: dict = {}
    for ln, module, st in _statements(datatb):
        low = st.lower()
        mparams = params
        m = re.match(r"parameter\s*\((.*)\)\s*$", low)
        if m:
            for a in _split_top(m.group(1)):
                k, v = a.split("=")
                params[k.strip()] = int(v)
            continue
        m = re.match(r"real\s*\(\s*kind\s*=\s*kind_phys\s*\)\s*,\s*parameter\s*::\s*(\w+)\s*=\s*([-+.\deE]+)", low)
        if m:
            real_params[(module, m.group(1))] = _parse_value(m.group(2), real4)[0]
            continue
        m = re.match(r"(real|integer)\b(.*?)::(.*)$", low)
        if m and module:
            kind, attrs, names = m.group(1), m.group(2), m.group(3)
            if "parameter" in attrs:
                continue
            dm = re.search(r"dimension\s*\(([^)]*)\)", attrs)
            common = _parse_dims(dm.group(1), mparams) if dm else None
            for item in _split_top(names):
                item = item.strip()
                if not item:
                    continue
                im = re.match(r"(\w+)\s*(?:\((.*)\))?\s*$", item)
                name = im.group(1)
                dims = _parse_dims(im.group(2), mparams) if im.group(2) else common
                if dims is None:
                    continue
                decls[(module, name)] = dims
                kinds[(module, name)] = kind
                size = int(np.prod([hi - lo + 1 for lo, hi in dims]))
                values[(module, name)] = np.full(size, np.nan)
                filled[(module, name)] = np.zeros(size, dtype=bool)
            continue
        m = re.match(r"data\s+(.*)$", st, flags=re.I | re.S)
        if m and module:
            body = m.group(1)
            # one or more  target / values /  groups
            for tm in re.finditer(r"([A-Za-z_]\w*)\s*(\([^/]*\))?\s*/([^/]*)/", body):
                name = tm.group(1).lower()
                sub = tm.group(2)
                vals = []
                for tok in tm.group(3).split(","):
                    if tok.strip():
                        vals.extend(_parse_value(tok, real4 and kinds[(module, name)] == "real"))
                key = (module, name)
                dims = decls[key]
                if sub:
                    subs = _split_top(sub.strip()[1:-1])
                    ranges = []
                    for s, (lo, hi) in zip(subs, dims):
                        s = s.strip()
                        if s == ":":
                            ranges.append(range(lo, hi + 1))
                        elif ":" in s:
                            a, b = s.split(":")
                            ranges.append(range(_eval_int(a, mparams), _eval_int(b, mparams) + 1))
                        else:
                            v = _eval_int(s, mparams)
                            ranges.append(range(v, v + 1))
                else:
                    ranges = [range(lo, hi + 1) for lo, hi in dims]
                # Linear (column-major) index of every element of the section,
                # listed in Fortran element order (first subscript fastest).
                grids = np.meshgrid(*[np.array(list(r), dtype=np.int64) for r in ranges],
                                    indexing="ij")
                lin = np.zeros(grids[0].shape, dtype=np.int64)
                stride = 1
                for g, (lo, hi) in zip(grids, dims):
                    lin += (g - lo) * stride
                    stride *= hi - lo + 1
                flat = lin.reshape(-1, order="F")
                if len(vals) != flat.size:
                    raise ValueError(f"{datatb}:{ln}: {name} expects {flat.size} values, got {len(vals)}")
                if filled[key][flat].any():
                    raise ValueError(f"{datatb}:{ln}: {name} element assigned twice")
                values[key][flat] = vals
                filled[key][flat] = True
                src_lines.setdefault(key, []).append(ln)
    return params, decls, kinds, values, filled, real_params, src_lines


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("ref_root")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--default-real-4", action="store_true")
    a = ap.parse_args(argv)
    params, decls, kinds, values, filled, real_params, src_lines = extract(a.ref_root, a.default_real_4)

    entries = []
    def add(module, name, cname):
        key = (module, name)
        if key not in values:
            return
        if not filled[key].all():
            raise ValueError(f"{module}:{name} has {int((~filled[key]).sum())} unassigned elements")
        entries.append((cname, module, name, decls[key], values[key], src_lines[key][0]))

    add("module_radlw_avplank", "totplnk", "totplnk")
    for nm in ("pref", "preflog", "tref", "chi_mls"):
        add("module_radlw_ref", nm, nm)
    for nm in ("absliq1", "absice0", "absice1", "absice2", "absice3", "ipat"):
        add("module_radlw_cldprlw", nm, nm)
    for b in range(1, 17):
        mod = f"module_radlw_kgb{b:02d}"
        for nm in _BAND_ARRAYS:
            add(mod, nm, f"b{b:02d}_{nm}")

    off = 0
    blob = bytearray()
    lines = []
    for cname, module, name, dims, vals, ln in entries:
        # 8-double alignment for every array
        pad = (-off) % 8
        blob += struct.pack(f"<{pad}d", *([0.0] * pad))
        off += pad
        ext = [hi - lo + 1 for lo, hi in dims]
        lines.append((cname, module, name, off, ext, dims, ln))
        blob += struct.pack(f"<{vals.size}d", *vals.tolist())
        off += vals.size
    sha = hashlib.sha256(bytes(blob)).hexdigest()

    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, "rrtmg_lw_tables.bin"), "wb") as fh:
        fh.write(bytes(blob))
    hdr = [
        "/* Generated by extract_tables.py from radlw_datatb.f (module_radlw_avplank,",
        " * module_radlw_ref, module_radlw_cldprlw, module_radlw_kgb01..16).",
        " * Offsets are in doubles into rrtmg_lw_tables.bin; each array is stored in",
        " * Fortran order (first index fastest). Do not edit. */",
        "#pragma once",
        f"#define RRTMG_LW_TABLES_NDOUBLE {off}",
        f"#define RRTMG_LW_TABLES_SHA256 \"{sha}\"",
        "namespace lwtab {",
    ]
    for cname, module, name, o, ext, dims, ln in lines:
        hdr.append(f"constexpr int {cname} = {o};  /* {name}{tuple(ext)} radlw_datatb.f:{ln} */")
    hdr.append("}  // namespace lwtab")
    hdr.append("")
    with open(os.path.join(a.out, "rrtmg_lw_table_layout.h"), "w") as fh:
        fh.write("\n".join(hdr))
    manifest = {
        "sha256": sha, "ndouble": off,
        "arrays": {c: {"module": m, "name": n, "offset": o, "shape": e, "line": ln}
                   for c, m, n, o, e, d, ln in lines},
        "real_parameters": {f"{m}:{n}": v for (m, n), v in real_params.items()},
    }
    with open(os.path.join(a.out, "rrtmg_lw_tables.json"), "w") as fh:
        json.dump(manifest, fh, indent=1, sort_keys=True)
    print(f"wrote {len(lines)} arrays, {off} doubles, sha256 {sha}")


if __name__ == "__main__":
    sys.exit(main())
