"""CPU-side checks of the C ABI: the CUDA library loads without a GPU and
exports every function declared in include/*.h; host-side validation paths
return errors instead of crashing."""
import ctypes as C
import glob
import os
import re

import pytest

from ccpp_physics_b200 import abi, synthetic

ROOT = os.path.join(os.path.dirname(__file__), "..")


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|void)\s+(rrtmg_[ls]w_gpu_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_header_symbols():
    from ccpp_physics_b200 import rrtmg_lw as lw
    L = lw.lib()
    declared = _declared()
    assert {"rrtmg_lw_gpu_init", "rrtmg_lw_gpu_run", "rrtmg_lw_gpu_run_ex", "rrtmg_sw_gpu_init",
            "rrtmg_sw_gpu_run", "rrtmg_sw_gpu_run_ex"} <= declared
    for n in sorted(declared):
        assert hasattr(L, n), n


def test_struct_layout_matches_header(tmp_path):
    """ctypes mirror == C header: sizeof and every field offset, from gcc."""
    import shutil
    import subprocess
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    structs = {"rrtmg_lw_run_args": abi.RunArgs, "rrtmg_lw_init_args": abi.InitArgs,
               "rrtmg_lw_exec": abi.ExecArgs, "rrtmg_lw_tuning": abi.Tuning,
               "rrtmg_lw_seed_args": abi.SeedArgs, "rrtmg_lw_overlap_args": abi.OverlapArgs,
               "rrtmg_lw_post_args": abi.PostArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rrtmg_lw_gpu.h"', 'int main(void){']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_run_before_init_reports_error():
    import numpy as np
    from ccpp_physics_b200 import rrtmg_lw as lw, synthetic
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("checks the no-GPU path")
    except ImportError:
        pass
    prof = synthetic.make_profiles(2, 10, seed=1)
    msg, err = lw.run_profile(prof, abi.alloc_outputs(2, 10))
    assert err == 1 and "init" in msg
    rc, msg = lw.rlwinit()
    assert rc == 1 and "CUDA" in msg


def test_block_args_offsets():
    """Physics blocks as views into one profile: every pointer moves to the
    block's first column; records move by their record size; ldim = npts."""
    import ctypes as C
    from ccpp_physics_b200 import rrtmg_lw as lw
    npts, nlay = 40, 20
    p = synthetic.make_profiles(npts, nlay, seed=1)
    o = abi.alloc_outputs(npts, nlay, hlw0=True, hlwb=True, flxprf=True)
    arr, keep = lw.block_args(p, o, [10, 25, 5])
    addr = lambda a, n: C.cast(getattr(a, n), C.c_void_p).value
    assert [a.npts for a in arr] == [10, 25, 5] and all(a.ldim == npts for a in arr)
    for name, step in (("plyr", 8), ("aeraod", 8), ("hlwb", 8), ("icseed", 4), ("topflx", 16),
                       ("sfcflx", 32), ("flxprf", 32)):
        assert addr(arr[1], name) - addr(arr[0], name) == 10 * step, name
        assert addr(arr[2], name) - addr(arr[0], name) == 35 * step, name
    with pytest.raises(ValueError):
        lw.block_args(p, o, [10, 10])


def test_packed_blocks_layout():
    """Blocks held as separate arrays: pack/unpack round-trip, each block's
    field is its own contiguous (n_b, ...) Fortran array, and block_args
    points each block at its segment with ldim = its column count."""
    import ctypes as C
    import numpy as np
    import torch
    from ccpp_physics_b200 import rrtmg_lw as lw
    npts, nlay, sizes = 40, 20, [10, 25, 5]
    p = {k: (torch.from_numpy(v) if isinstance(v, np.ndarray) else v)
         for k, v in synthetic.make_profiles(npts, nlay, seed=1).items()}
    o = {k: torch.from_numpy(v) for k, v in abi.alloc_outputs(npts, nlay, hlw0=True, hlwb=True,
                                                               flxprf=True).items()}
    for k in o:
        o[k].copy_(torch.arange(o[k].numel(), dtype=o[k].dtype).view(o[k].shape))
    pp, po = lw.pack_blocks(p, sizes), lw.pack_blocks(o, sizes)
    for src, packed in ((p, pp), (o, po)):
        back = lw.unpack_blocks(packed)
        for k, v in src.items():
            if isinstance(v, torch.Tensor):
                assert torch.equal(back[k], v), k
    # block 1 (columns 10..34) of an (nlay, npts) field and of the (nlay+1, npts, 4) records
    seg = pp["plyr"].reshape(-1)[nlay * 10: nlay * 35].view(nlay, 25)
    assert torch.equal(seg, p["plyr"][:, 10:35])
    seg = po["flxprf"].reshape(-1)[(nlay + 1) * 4 * 10: (nlay + 1) * 4 * 35].view(nlay + 1, 25, 4)
    assert torch.equal(seg, o["flxprf"][:, 10:35])
    arr, keep = lw.block_args(pp, po, sizes)
    addr = lambda a, n: C.cast(getattr(a, n), C.c_void_p).value
    assert [a.ldim for a in arr] == sizes
    for name, per_col in (("plyr", 8 * nlay), ("aeraod", 8 * nlay * 16), ("icseed", 4), ("topflx", 16),
                          ("flxprf", 32 * (nlay + 1)), ("hlwb", 8 * nlay * 16)):
        assert addr(arr[1], name) - addr(arr[0], name) == 10 * per_col, name
        assert addr(arr[2], name) - addr(arr[0], name) == 35 * per_col, name
    with pytest.raises(ValueError):
        lw.block_args(pp, o, sizes)          # profile packed, outputs not


def test_fortran_shims_match_the_c_abi():
    """No Fortran compiler here, so the shims are checked as text: every
    bind(c) name is a function declared in include/*.h and exported, and every
    bind(c) record has the C struct's fields in order with matching kinds
    (the ctypes mirrors are pinned to the header by the gcc layout tests)."""
    from ccpp_physics_b200 import rrtmg_lw as lw, rrtmg_sw as sw
    L = lw.lib()
    declared = _declared()
    mirrors = {"c_init_args": abi.InitArgs, "c_run_args": abi.RunArgs, "c_sw_init_args": sw.SwInitArgs,
               "c_sw_run_args": sw.SwRunArgs, "c_sw_exec": sw.SwExec, "c_sw_pre_args": sw.SwPreArgs,
               "c_sw_post_args": sw.SwPostArgs, "c_lw_exec": abi.ExecArgs, "c_lw_post_args": abi.PostArgs}
    kinds = {"integer(c_int32_t)": C.c_int32, "real(c_double)": C.c_double}
    seen = set()
    for path in sorted(glob.glob(os.path.join(ROOT, "ccpp_physics_b200", "fortran", "*.F90"))):
        txt = open(path).read()
        for name in re.findall(r'bind\(c,\s*name="(\w+)"\)', txt):
            assert name in declared and hasattr(L, name), (path, name)
        for tname, body in re.findall(r"type, bind\(c\) :: (\w+)\n(.*?)\n\s*end type", txt, re.S):
            fields = []
            for line in body.splitlines():
                kind, names = (p.strip() for p in line.split("::"))
                for n in names.split(","):
                    fields.append((n.split("=")[0].strip(), kind))
            py = mirrors[tname]._fields_
            assert [f for f, _ in fields] == [f for f, _ in py], (path, tname)
            for (f, kind), (_, ct) in zip(fields, py):
                if kind == "type(c_ptr)":
                    assert issubclass(ct, (C._Pointer, C.c_void_p)), (tname, f)
                else:
                    assert kinds[kind] is ct, (tname, f)
            seen.add(tname)
    assert seen == set(mirrors)
