"""Python mirror of the Fortran ``rrtmg_lw`` module interface, on the GPU.

``rlwinit`` and ``rrtmg_lw_run`` keep the argument names, meanings and error
convention of physics/Radiation/RRTMG/radlw_main.F90 (rlwinit :1322-1324,
rrtmg_lw_run :419-434): outputs are caller-owned arrays filled in place and
the functions return ``(errmsg, errflg)``.  Arrays are Fortran-ordered
``(npts, nlay[, nbands])`` fields, i.e. C-contiguous ``(nlay, npts)`` numpy
arrays (host memory) or torch CUDA tensors (device memory).

There is no CPU fallback: every call goes through ``librrtmg_lw_gpu.so``
(include/rrtmg_lw_gpu.h), and importing this module raises if the library is
missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "librrtmg_lw_gpu.so")
_lib = None

PRECISIONS = {"fp64": abi.FP64, "fp32": abi.FP32, "surrogate": abi.SURROGATE}


class RRTMGLWError(RuntimeError):
    pass


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                              f"(make -C ccpp_physics_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        L.rrtmg_lw_gpu_init.argtypes = [C.POINTER(abi.InitArgs), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_run.argtypes = [C.POINTER(abi.RunArgs), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_run_ex.argtypes = [C.POINTER(abi.RunArgs), C.POINTER(abi.ExecArgs), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_mcica.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32] + [C.c_void_p] * 7 + \
            [C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_gas_optics.argtypes = [C.POINTER(abi.RunArgs), C.c_int32, C.c_void_p, C.c_void_p,
                                              C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_run_blocks.argtypes = [C.POINTER(abi.RunArgs), C.c_int32, C.POINTER(abi.ExecArgs),
                                              C.POINTER(abi.Tuning), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_set_tuning.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_autotune.argtypes = [C.POINTER(abi.RunArgs), C.c_int32, C.c_int32, C.c_void_p,
                                            C.c_int64, C.POINTER(abi.Tuning), C.POINTER(C.c_float),
                                            C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_seeds.argtypes = [C.POINTER(abi.SeedArgs), C.POINTER(abi.ExecArgs), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_overlap_params.argtypes = [C.POINTER(abi.OverlapArgs), C.POINTER(abi.ExecArgs),
                                                  C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_post.argtypes = [C.POINTER(abi.PostArgs), C.POINTER(abi.ExecArgs), C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_finalize.argtypes = []
        _lib = L
    return _lib


def rlwinit(me=1, rad_hr_units=1, inc_minor_gas=True, ilwcliq=1, isubclw=2, iovr=1,
            iovr_rand=0, iovr_maxrand=1, iovr_max=2, iovr_dcorr=3, iovr_exp=4, iovr_exprand=5,
            device=0):
    """rlwinit (radlw_main.F90:1322): returns (errflg, errmsg)."""
    ia = abi.make_init_args(me=me, rad_hr_units=rad_hr_units, inc_minor_gas=inc_minor_gas,
                            ilwcliq=ilwcliq, isubclw=isubclw, iovr=iovr, device=device,
                            iovr_rand=iovr_rand, iovr_maxrand=iovr_maxrand, iovr_max=iovr_max,
                            iovr_dcorr=iovr_dcorr, iovr_exp=iovr_exp, iovr_exprand=iovr_exprand)
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_init(C.byref(ia), msg, 512)
    return rc, msg.value.decode()


def _is_device(x):
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except ImportError:
        return False


def torch_stream(stream, x):
    """The CUDA stream to run on: `stream` if given, else torch's current
    stream of device tensor `x` (so library work is ordered after the torch
    work that produced its inputs), else None (host data)."""
    if stream is not None:
        return stream
    if _is_device(x):
        import torch
        h = torch.cuda.current_stream(x.device).cuda_stream
        return h or None
    return None


def run_profile(prof: dict, out: dict, *, precision="fp64", flags=None, stream=None, sync=True):
    """rrtmg_lw_run over a profile dict (field name -> array) into ``out``.
    Returns (errmsg, errflg) like the Fortran routine."""
    keep = []
    a = abi.make_run_args(prof, out, flags=flags, keep=keep)
    device = _is_device(prof["plyr"])
    stream = torch_stream(stream, prof["plyr"])
    x = abi.ExecArgs(precision=PRECISIONS[precision] if isinstance(precision, str) else precision,
                     memory=abi.DEVICE if device else abi.HOST,
                     stream=None if stream is None else C.c_void_p(stream), sync=int(sync))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_run_ex(C.byref(a), C.byref(x), msg, 512)
    return msg.value.decode(), rc


def rrtmg_lw_run(plyr, plvl, tlyr, tlvl, qlyr, olyr, gasvmr_co2, gasvmr_n2o, gasvmr_ch4, gasvmr_o2,
                 gasvmr_co, gasvmr_cfc11, gasvmr_cfc12, gasvmr_cfc22, gasvmr_ccl4, icseed, aeraod,
                 aerssa, sfemis, sfgtmp, dzlyr, delpin, de_lgth, alpha, npts, nlay, nlp1, lprnt, cld_cf,
                 lslwr, top_at_1, iovr, iovr_rand, iovr_maxrand, iovr_max, iovr_dcorr, iovr_exp,
                 iovr_exprand, inc_minor_gas, ilwcliq, ilwcice, isubclw, hlwc, topflx, sfcflx, cldtau,
                 hlw0=None, hlwb=None, flxprf=None, cld_lwp=None, cld_ref_liq=None, cld_iwp=None,
                 cld_ref_ice=None, cld_rwp=None, cld_ref_rain=None, cld_swp=None, cld_ref_snow=None,
                 cld_od=None, *, precision="fp64", stream=None):
    """rrtmg_lw_run (radlw_main.F90:419) with the reference's argument list.
    Returns (errmsg, errflg)."""
    if nlp1 != nlay + 1:
        return "rrtmg_lw_run: nlp1 must equal nlay+1", 1
    prof = dict(npts=npts, nlay=nlay, flags=dict(
        lprnt=int(lprnt), lslwr=int(lslwr), top_at_1=int(top_at_1), inc_minor_gas=int(inc_minor_gas),
        iovr=iovr, iovr_rand=iovr_rand, iovr_maxrand=iovr_maxrand, iovr_max=iovr_max,
        iovr_dcorr=iovr_dcorr, iovr_exp=iovr_exp, iovr_exprand=iovr_exprand, ilwcliq=ilwcliq,
        ilwcice=ilwcice, isubclw=isubclw))
    loc = dict(locals())
    for n in abi.INPUT_FIELDS + ("icseed", "aeraod", "aerssa", "sfemis", "sfgtmp", "dzlyr", "delpin",
                                 "de_lgth", "alpha", "cld_cf") + abi.OPTIONAL_CLOUD_FIELDS:
        prof[n] = loc[n]
    out = {n: loc[n] for n in abi.OUTPUT_FIELDS + abi.OPTIONAL_OUTPUT_FIELDS if loc[n] is not None}
    return run_profile(prof, out, precision=precision, stream=stream)


def mcica_bits(cldf, seed, iovr=1, dz=None, de_lgth=None, alpha=None, stream=None):
    """Sub-column cloud flags of ``mcica_subcol`` on the GPU for device
    tensors cldf (nlay, npts) float64 and seed (npts,) int32; iovr 3 also
    takes dz (nlay, npts) [km] and de_lgth (npts,) [km], iovr 4/5 alpha
    (nlay, npts).  Returns a (npts, 140, nwords) int32 tensor of bit words
    (bit k&31 of word k>>5)."""
    import torch
    nlay, npts = cldf.shape
    nw = (nlay + 31) // 32
    stream = torch_stream(stream, cldf)
    bits = torch.zeros((npts, abi.NGPT, nw), dtype=torch.int32, device=cldf.device)
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_mcica(npts, nlay, npts, iovr, ptr(seed), ptr(cldf), ptr(dz), ptr(de_lgth), ptr(alpha),
                                  C.c_void_p(bits.data_ptr()), stream, msg, 512)
    if rc:
        raise RRTMGLWError(msg.value.decode())
    return bits


def gas_optics(prof: dict, precision="fp64", stream=None):
    """setcoef + taumol on the GPU for a device-resident profile dict.
    Returns (taug, fracs) float64 tensors of shape (npts, nlay, 140), layers
    surface first (the internal order of the reference)."""
    import torch
    npts, nlay = prof["npts"], prof["nlay"]
    taug = torch.empty((npts, nlay, abi.NGPT), dtype=torch.float64, device=prof["plyr"].device)
    fracs = torch.empty_like(taug)
    keep = []
    a = abi.make_run_args(prof, {}, keep=keep)
    stream = torch_stream(stream, prof["plyr"])
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_gas_optics(C.byref(a), PRECISIONS[precision], C.c_void_p(taug.data_ptr()),
                                       C.c_void_p(fracs.data_ptr()), stream, msg, 512)
    if rc:
        raise RRTMGLWError(msg.value.decode())
    return taug, fracs


# column axis of the fields whose columns are not the last axis (records)
_COL_AXIS = {"topflx": 0, "sfcflx": 0, "flxprf": 1}


def _block_index(sizes, A, R, device):
    """Per column: first packed element of its block and its block size."""
    import torch
    sizes_t = torch.as_tensor(np.asarray(sizes, dtype=np.int64), device=device)
    c0 = torch.cumsum(sizes_t, 0) - sizes_t
    n_col = torch.repeat_interleave(sizes_t, sizes_t)
    c0_col = torch.repeat_interleave(c0, sizes_t)
    j = torch.arange(int(sizes_t.sum()), device=device) - c0_col
    return (A * c0_col + j) * R, n_col * R


def _pack_field(v, axis, sizes, unpack=False, full=None):
    """Block-packed copy of field v (or, with unpack, v's columns scattered
    back into ``full``): block b's columns become one contiguous
    (n_b, ...) Fortran array."""
    import torch
    npts = v.shape[axis] if not unpack else full.shape[axis]
    shape = (full if unpack else v).shape
    A = int(np.prod(shape[:axis])) if axis > 0 else 1
    R = int(np.prod(shape[axis + 1:])) if axis + 1 < len(shape) else 1
    src = (full if unpack else v).reshape(A, npts, R)
    base, step = _block_index(sizes, A, R, src.device)
    dst = torch.empty_like(src) if not unpack else None
    flat = (dst if not unpack else v).reshape(-1)
    r = torch.arange(R, device=src.device)
    rows = max(1, (1 << 27) // max(1, npts * R))       # index chunks of <= 128 M elements
    for a0 in range(0, A, rows):
        a = torch.arange(a0, min(A, a0 + rows), device=src.device)
        idx = (base[None, :, None] + a[:, None, None] * step[None, :, None] + r[None, None, :]).reshape(-1)
        if unpack:
            src[a0:a0 + len(a)] = flat[idx].view(len(a), npts, R)
        else:
            flat.index_copy_(0, idx, src[a0:a0 + len(a)].reshape(-1))
    return dst.view(shape) if not unpack else full


def pack_blocks(d: dict, sizes, *, inplace=False) -> dict:
    """A copy of a Fortran-ordered profile or output dict (device tensors) in
    which every physics block of ``sizes`` columns is its own contiguous
    (n_b, ...) array, the way a host that allocates each block separately
    (ccpp-physics' GFS blocks) holds them.  Tensors keep their shapes; only
    the element order changes.  block_args/run_blocks recognise the layout.
    With inplace, d itself is converted field by field (one field's extra
    memory at a time) and returned."""
    import torch
    out = d if inplace else {k: v for k, v in d.items() if not isinstance(v, torch.Tensor)}
    for k in [k for k, v in d.items() if isinstance(v, torch.Tensor)]:
        v = d[k]
        packed = _pack_field(v, _COL_AXIS.get(k, v.dim() - 1), sizes)
        if inplace:
            d[k] = None
            del v
        out[k] = packed
    out["_packed_sizes"] = np.asarray(sizes, dtype=np.int64)
    return out


def unpack_blocks(d: dict) -> dict:
    """Inverse of pack_blocks: tensors in the ordinary column layout."""
    import torch
    sizes = d["_packed_sizes"]
    out = {k: v for k, v in d.items() if not isinstance(v, torch.Tensor) and k != "_packed_sizes"}
    for k, v in d.items():
        if isinstance(v, torch.Tensor):
            out[k] = _pack_field(v, _COL_AXIS.get(k, v.dim() - 1), sizes, unpack=True, full=torch.empty_like(v))
    return out


def block_args(prof: dict, out: dict, sizes, *, flags=None):
    """RunArgs array describing consecutive physics blocks of ``sizes``
    columns.  For an ordinary profile/output dict each block is a view into
    the full arrays (it points at its first column and uses the full column
    count as ldim, the way a host passes slices of larger arrays); for a dict
    from pack_blocks each block is its own contiguous array with ldim = its
    column count."""
    keep = []
    base = abi.make_run_args(prof, out, flags=flags, keep=keep)
    npts = prof["npts"]
    if int(np.sum(sizes)) != npts:
        raise ValueError("block sizes must add up to npts")
    packed = "_packed_sizes" in prof
    if packed != ("_packed_sizes" in out) or (packed and not np.array_equal(prof["_packed_sizes"], sizes)):
        raise ValueError("profile and outputs must share the block packing of sizes")
    arr = (abi.RunArgs * len(sizes))()
    col_fields = set(abi.INPUT_FIELDS + ("aeraod", "aerssa", "sfemis", "sfgtmp", "dzlyr", "delpin",
                                         "de_lgth", "alpha", "cld_cf") + abi.OPTIONAL_CLOUD_FIELDS +
                     ("hlwc", "cldtau", "hlw0", "hlwb"))
    rec = {"topflx": 2, "sfcflx": 4, "flxprf": 4}
    per_col = {}          # bytes of one column of each field (packed layout)
    if packed:
        for name, _ in abi.RunArgs._fields_:
            t = prof.get(name, out.get(name))
            if t is not None and hasattr(t, "numel"):
                per_col[name] = t.numel() // npts * t.element_size()
    c0 = 0
    for b, n in enumerate(sizes):
        a = abi.RunArgs.from_buffer_copy(base)
        a.npts, a.ldim = int(n), (int(n) if packed else npts)
        for name, _ in abi.RunArgs._fields_:
            p = getattr(a, name)
            if not isinstance(p, C._Pointer) or not p:
                continue
            addr = C.cast(p, C.c_void_p).value
            if packed:
                off = per_col[name] * c0
            elif name == "icseed":
                off = 4 * c0
            elif name in rec:
                off = 8 * rec[name] * c0
            elif name in col_fields:
                off = 8 * c0
            else:
                continue
            setattr(a, name, C.cast(C.c_void_p(addr + off), type(p)))
        arr[b] = a
        c0 += int(n)
    return arr, keep


def run_blocks(prof: dict, out: dict, sizes, *, precision="fp64", tuning=None, stream=None, sync=True,
               kernel_ms=None):
    """All physics blocks of ``sizes`` columns (views into one device-resident
    profile) in one call of rrtmg_lw_gpu_run_blocks.  ``tuning``: an
    abi.Tuning or dict (rt_warps, gas_per_sm, chunk_cols, use_graph).
    Returns (errmsg, errflg)."""
    arr, keep = block_args(prof, out, sizes)
    stream = torch_stream(stream, prof["plyr"])
    x = abi.ExecArgs(precision=PRECISIONS[precision] if isinstance(precision, str) else precision,
                     memory=abi.DEVICE, stream=None if stream is None else C.c_void_p(stream), sync=int(sync))
    if kernel_ms is not None:
        x.kernel_ms = kernel_ms
    t = abi.Tuning(**tuning) if isinstance(tuning, dict) else tuning
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_run_blocks(arr, len(arr), C.byref(x), C.byref(t) if t is not None else None, msg, 512)
    return msg.value.decode(), rc


def tuning_key(nlay: int, precision: str, device_name: str) -> str:
    """Key of a launch shape in the autotuner's JSON cache: the kernels'
    shape depends on the layer count (layers per lane), the precision and
    the GPU."""
    return f"{device_name}|nlay={int(nlay)}|{precision}"


def set_tuning(nlay: int, precision: str, tuning):
    """Default launch shape of later calls with this layer count and
    precision (rrtmg_lw_gpu_set_tuning); None clears it."""
    t = None if tuning is None else abi.Tuning(**{n: int(tuning.get(n, 0)) for n, _ in abi.Tuning._fields_})
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_set_tuning(int(nlay), PRECISIONS[precision], None if t is None else C.byref(t), msg, 512)
    if rc:
        raise RRTMGLWError(msg.value.decode())


def autotune(prof: dict, out: dict, sizes, *, precision="fp32", sample_cols=0, stream=None, cache=None,
             device_name=None):
    """Autotune the launch shape on the physics blocks of ``sizes`` columns;
    returns (tuning dict, ms per call).

    cache: path of a JSON file of chosen shapes keyed by (GPU, layer count,
    precision).  A hit sets that shape as the default of later calls
    (set_tuning) without timing and returns (tuning, ms recorded when it was
    chosen); a miss times the candidates and adds the choice to the file."""
    nlay = int(prof["nlay"])
    key = None
    if cache is not None:
        if device_name is None:
            import torch
            device_name = torch.cuda.get_device_name(prof["plyr"].device) if hasattr(prof["plyr"], "device") \
                else torch.cuda.get_device_name()
        key = tuning_key(nlay, precision, device_name)
        table = _read_tuning_cache(cache)
        if key in table:
            hit = table[key]
            set_tuning(nlay, precision, hit["tuning"])
            return dict(hit["tuning"]), float(hit["ms"])
    arr, keep = block_args(prof, out, sizes)
    stream = torch_stream(stream, prof["plyr"])
    best = abi.Tuning()
    ms = C.c_float(0.0)
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_autotune(arr, len(arr), PRECISIONS[precision], None if stream is None else
                                     C.c_void_p(stream), int(sample_cols), C.byref(best), C.byref(ms), msg, 512)
    if rc:
        raise RRTMGLWError(msg.value.decode())
    tuning = {n: getattr(best, n) for n, _ in abi.Tuning._fields_}
    if key is not None:
        table = _read_tuning_cache(cache)
        table[key] = {"tuning": tuning, "ms": float(ms.value)}
        _write_tuning_cache(cache, table)
    return tuning, ms.value


def _read_tuning_cache(path) -> dict:
    import json
    try:
        with open(path) as fh:
            table = json.load(fh)
    except FileNotFoundError:
        return {}
    if not isinstance(table, dict):
        raise RRTMGLWError(f"{path}: not a tuning cache (a JSON object is expected)")
    return table


def _write_tuning_cache(path, table: dict):
    import json
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as fh:
        json.dump(table, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)   # readers never see a half-written file


def to_device(prof: dict, device="cuda"):
    """Copy a numpy profile dict to device tensors (Fortran layout kept)."""
    import torch
    out = dict(npts=prof["npts"], nlay=prof["nlay"], flags=dict(prof["flags"]))
    for k, v in prof.items():
        if isinstance(v, np.ndarray):
            out[k] = torch.from_numpy(v).to(device)
    return out
