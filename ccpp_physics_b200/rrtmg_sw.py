"""Host-side mirror of the RRTMG-SW entry points (``include/rrtmg_sw_gpu.h``).

``rswinit`` and ``rrtmg_sw_run`` keep the argument names and meaning of the
Fortran module ``rrtmg_sw`` (physics/Radiation/RRTMG/radsw_main.F90:493-510,
1388-1390); both call the CUDA library ``librrtmg_lw_gpu.so`` (the longwave
and shortwave paths share one library) through its C ABI.  There is no CPU
fallback: the calls fail loudly when the library or a GPU is missing.

Arrays are Fortran-ordered (column index fastest): a field of shape
``(npts, nlay)`` is a C-contiguous numpy/torch array of shape
``(nlay, npts)``; aerosol fields ``(npts, nlay, 14)`` are ``(14, nlay, npts)``.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import abi
from .synthetic import _uniform

NBANDS = 14
NGPT = 112

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

INPUT_FIELDS = abi.INPUT_FIELDS
OPTIONAL_CLOUD_FIELDS = ("cld_lwp", "cld_ref_liq", "cld_iwp", "cld_ref_ice", "cld_rwp", "cld_ref_rain",
                         "cld_swp", "cld_ref_snow", "cld_od", "cld_ssa", "cld_asy")
OUTPUT_FIELDS = ("hswc", "topflx", "sfcflx", "cldtau")
OPTIONAL_OUTPUT_FIELDS = ("hsw0", "hswb", "flxprf", "fdncmp")

DEFAULT_FLAGS = dict(lprnt=0, lsswr=1, top_at_1=0, inc_minor_gas=1, iovr=1, iswcliq=1, iswcice=3,
                     isubcsw=2, iswmode=2)


class SwInitArgs(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "me", "rad_hr_units", "inc_minor_gas", "iswcliq", "isubcsw", "iovr", "iovr_rand", "iovr_maxrand",
        "iovr_max", "iovr_dcorr", "iovr_exp", "iovr_exprand", "iswmode", "device")]


class SwRunArgs(C.Structure):
    _fields_ = (
        [(n, C.c_int32) for n in ("npts", "nlay", "nlp1", "ldim", "nday", "lprnt", "lsswr", "top_at_1",
                                  "inc_minor_gas", "iovr", "iovr_rand", "iovr_maxrand", "iovr_max",
                                  "iovr_dcorr", "iovr_exp", "iovr_exprand", "iswcliq", "iswcice",
                                  "isubcsw", "iswmode")]
        + [("solcon", C.c_double)]
        + [(n, _dp) for n in INPUT_FIELDS]
        + [("icseed", _ip), ("idxday", _ip)]
        + [(n, _dp) for n in ("aeraod", "aerssa", "aerasy", "sfcalb_nir_dir", "sfcalb_nir_dif",
                              "sfcalb_uvis_dir", "sfcalb_uvis_dif", "dzlyr", "delpin", "de_lgth", "alpha",
                              "cosz", "cld_cf")]
        + [(n, _dp) for n in OPTIONAL_CLOUD_FIELDS]
        + [(n, _dp) for n in OUTPUT_FIELDS + OPTIONAL_OUTPUT_FIELDS]
    )


class SwExec(C.Structure):
    _fields_ = [("precision", C.c_int32), ("memory", C.c_int32), ("stream", C.c_void_p),
                ("sync", C.c_int32), ("reserved", C.c_int32), ("kernel_ms", C.POINTER(C.c_float))]


class SwPreArgs(C.Structure):
    """rrtmg_sw_pre_args: rad_sw_pre_run (rad_sw_pre.F90:14-51)."""
    _fields_ = [("im", C.c_int32), ("lsswr", C.c_int32), ("coszen", _dp), ("nday", _ip), ("idxday", _ip)]


POST_INPUT_FIELDS = ("sfcalb1", "sfcalb2", "sfcalb3", "sfcalb4", "htswc", "htsw0")
POST_OUTPUT_FIELDS = ("nirbmdi", "nirdfdi", "visbmdi", "visdfdi", "nirbmui", "nirdfui", "visbmui", "visdfui",
                      "sfcdsw", "sfcnsw", "htrsw", "swhc", "scmpsw", "sfcfsw", "topfsw")


class SwPostArgs(C.Structure):
    """rrtmg_sw_post_args: rrtmg_sw_post_run (rrtmg_sw_post.F90:13-129)."""
    _fields_ = ([(n, C.c_int32) for n in ("im", "levr", "levs", "ltp", "nday", "lm", "kd", "lsswr", "swhtr")]
                + [(n, _dp) for n in POST_INPUT_FIELDS + POST_OUTPUT_FIELDS])


def make_init_args(rad_hr_units=1, inc_minor_gas=True, iswcliq=1, isubcsw=2, iovr=1, iswmode=2, me=1,
                   device=0) -> SwInitArgs:
    return SwInitArgs(me=me, rad_hr_units=rad_hr_units, inc_minor_gas=int(inc_minor_gas), iswcliq=iswcliq,
                      isubcsw=isubcsw, iovr=iovr, iswmode=iswmode, device=device, **abi.OVERLAP_FLAGS)


def add_sw_inputs(prof: dict, *, seed: int = 1, col_offset: int = 0, night_fraction: float = 0.0,
                  aerosol: bool = True, precip: bool = False) -> dict:
    """Add the shortwave-only inputs to a profile of ``synthetic.make_profiles``
    (same counter-based hashing, so a column's values depend only on its
    global index):

    * cos(solar zenith) ~ U(0.05, 1); a column is night (cosz = 0, left out
      of idxday) with probability ``night_fraction``;
    * surface albedos (near-IR / UV+visible, direct / diffuse) ~ U(0.05, 0.35);
    * aerosol optical depth per band and layer: 0.1 * exp(-z/2 km) * U(0, 1)
      * dz / 1 km, single-scattering albedo U(0.8, 1), asymmetry U(0.5, 0.8)
      (zero when ``aerosol`` is False);
    * rain and snow paths (``precip``): where there is cloud and T > 273 K a
      rain path LogN(ln 5, 1) g/m2 with re 500 um; snow LogN(ln 3, 1) with
      re U(20, 80) um where T < 263 K;
    * solar constant 1361 W/m2.
    """
    npts, nlay = prof["npts"], prof["nlay"]
    col = (torch.arange(npts, dtype=torch.int64) + col_offset).reshape(1, npts)
    lay = torch.arange(nlay, dtype=torch.int64).reshape(nlay, 1)
    cosz = (0.05 + 0.95 * _uniform(seed, col, 60))[0]
    night = _uniform(seed, col, 61)[0] < night_fraction
    cosz = torch.where(night, torch.zeros_like(cosz), cosz)
    out = dict(prof)
    out["cosz"] = cosz.numpy()
    out["idxday"] = (np.nonzero(~night.numpy())[0] + 1).astype(np.int32)
    out["solcon"] = 1361.0
    for i, n in enumerate(("sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir", "sfcalb_uvis_dif")):
        out[n] = (0.05 + 0.30 * _uniform(seed, col, 62 + i))[0].numpy()
    dz = torch.as_tensor(np.asarray(prof["dzlyr"]))
    z = torch.cumsum(dz, 0) - 0.5 * dz
    if aerosol:
        b = torch.arange(NBANDS, dtype=torch.int64).reshape(NBANDS, 1, 1)
        lb = lay.reshape(1, nlay, 1) * NBANDS + b
        c3 = col.reshape(1, 1, npts)
        aod = 0.1 * torch.exp(-z / 2.0).reshape(1, nlay, npts) * dz.reshape(1, nlay, npts) * _uniform(seed, c3, 70, lb)
        out["aeraod"] = aod.numpy().copy()
        out["aerssa"] = (0.8 + 0.2 * _uniform(seed, c3, 71, lb)).numpy().copy()
        out["aerasy"] = (0.5 + 0.3 * _uniform(seed, c3, 72, lb)).numpy().copy()
    else:
        for n in ("aeraod", "aerssa", "aerasy"):
            out[n] = np.zeros((NBANDS, nlay, npts))
    if precip:
        t = torch.as_tensor(np.asarray(prof["tlyr"]))
        cf = torch.as_tensor(np.asarray(prof["cld_cf"]))
        has = cf > 0.0
        rwp = torch.exp(math.log(5.0) + _normal_t(seed, col, 80, lay))
        swp = torch.exp(math.log(3.0) + _normal_t(seed, col, 82, lay))
        out["cld_rwp"] = torch.where(has & (t > 273.0), rwp, torch.zeros_like(rwp)).numpy()
        out["cld_ref_rain"] = np.full((nlay, npts), 500.0)
        out["cld_swp"] = torch.where(has & (t < 263.0), swp, torch.zeros_like(swp)).numpy()
        out["cld_ref_snow"] = (20.0 + 60.0 * _uniform(seed, col, 84, lay)).numpy()
    out["sw_flags"] = dict(DEFAULT_FLAGS)
    return out


def _normal_t(seed, col, field, layer):
    u1 = _uniform(seed, col, field, layer)
    u2 = _uniform(seed, col, field + 1000, layer)
    return torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * u2)


def alloc_outputs(npts, nlay, *, hsw0=True, hswb=False, flxprf=False, fdncmp=True, like=None):
    """Output arrays (numpy, or torch on ``like``'s device when given)."""
    def z(*shape):
        if like is not None:
            return torch.zeros(shape, dtype=torch.float64, device=like.device)
        return np.zeros(shape)
    out = dict(hswc=z(nlay, npts), topflx=z(npts, 3), sfcflx=z(npts, 4), cldtau=z(nlay, npts))
    if hsw0:
        out["hsw0"] = z(nlay, npts)
    if hswb:
        out["hswb"] = z(NBANDS, nlay, npts)
    if flxprf:
        out["flxprf"] = z(nlay + 1, npts, 4)
    if fdncmp:
        out["fdncmp"] = z(npts, 6)
    return out


def make_run_args(prof: dict, out: dict, *, flags: dict | None = None, keep=None, ldim: int = 0) -> SwRunArgs:
    """Fill SwRunArgs from a profile with SW inputs (``add_sw_inputs``) and
    output arrays.  ``keep`` collects converted arrays so they outlive the
    call; ``ldim`` > npts describes arrays that are slices of (ldim, ...)
    arrays."""
    keep = [] if keep is None else keep
    fl = dict(prof.get("sw_flags", DEFAULT_FLAGS))
    if flags:
        fl.update(flags)
    npts, nlay = prof["npts"], prof["nlay"]
    idx = prof["idxday"]
    a = SwRunArgs(npts=npts, nlay=nlay, nlp1=nlay + 1, ldim=ldim, nday=int(len(idx)), solcon=prof["solcon"],
                  **abi.OVERLAP_FLAGS)
    for k in ("lprnt", "lsswr", "top_at_1", "inc_minor_gas", "iovr", "iswcliq", "iswcice", "isubcsw", "iswmode"):
        setattr(a, k, int(fl[k]))
    for n in INPUT_FIELDS + ("aeraod", "aerssa", "aerasy", "sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir",
                             "sfcalb_uvis_dif", "dzlyr", "delpin", "de_lgth", "alpha", "cosz", "cld_cf"):
        setattr(a, n, _p(prof[n], keep, np.float64))
    if prof.get("icseed") is not None:      # isubcsw = 0, 1 draw no seeds from it
        a.icseed = _p(prof["icseed"], keep, np.int32)
    a.idxday = _p(idx, keep, np.int32)
    for n in OPTIONAL_CLOUD_FIELDS:
        if prof.get(n) is not None:
            setattr(a, n, _p(prof[n], keep, np.float64))
    for n in OUTPUT_FIELDS + OPTIONAL_OUTPUT_FIELDS:
        if out.get(n) is not None:
            setattr(a, n, _p(out[n], keep, np.float64))
    return a


def _p(x, keep, dtype):
    """Pointer to a numpy array (converted to a contiguous ``dtype`` copy
    when needed) or to a contiguous torch tensor's storage."""
    ctype = _dp if dtype == np.float64 else _ip
    if isinstance(x, torch.Tensor):
        if not x.is_contiguous():
            raise ValueError("torch arrays passed to rrtmg_sw_run must be contiguous")
        keep.append(x)
        return C.cast(C.c_void_p(x.data_ptr()), ctype)
    arr = np.ascontiguousarray(x, dtype=dtype)
    if arr is not x:
        keep.append(arr)
    else:
        keep.append(x)
    return arr.ctypes.data_as(ctype)


_lib = None


def lib():
    """The CUDA library with the SW entry points' signatures set."""
    global _lib
    if _lib is None:
        from . import rrtmg_lw
        L = rrtmg_lw.lib()
        L.rrtmg_sw_gpu_init.argtypes = [C.POINTER(SwInitArgs), C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_run.argtypes = [C.POINTER(SwRunArgs), C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_run_ex.argtypes = [C.POINTER(SwRunArgs), C.POINTER(SwExec), C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_gas_optics.argtypes = [C.POINTER(SwRunArgs)] + [C.c_void_p] * 4 + [C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_run_blocks.argtypes = [C.POINTER(SwRunArgs), C.c_int32, C.POINTER(SwExec), C.c_char_p,
                                              C.c_int32]
        L.rrtmg_sw_gpu_mcica.argtypes = ([C.c_int32] * 4 + [C.c_void_p] * 6 + [C.c_void_p, C.c_char_p, C.c_int32])
        L.rrtmg_sw_gpu_pre.argtypes = [C.POINTER(SwPreArgs), C.POINTER(SwExec), C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_post.argtypes = [C.POINTER(SwPostArgs), C.POINTER(SwExec), C.c_char_p, C.c_int32]
        L.rrtmg_sw_gpu_finalize.argtypes = []
        L.rrtmg_sw_gpu_finalize.restype = None
        _lib = L
    return _lib


class RrtmgSwError(RuntimeError):
    pass


def rswinit(me=1, rad_hr_units=1, inc_minor_gas=True, iswcliq=1, isubcsw=2, iovr=1, iswmode=2, device=0):
    """rswinit (radsw_main.F90:1388): returns nothing, raises on errflg."""
    a = make_init_args(rad_hr_units, inc_minor_gas, iswcliq, isubcsw, iovr, iswmode, me, device)
    msg = C.create_string_buffer(512)
    if lib().rrtmg_sw_gpu_init(C.byref(a), msg, 512):
        raise RrtmgSwError(msg.value.decode())


def rrtmg_sw_run(prof: dict, out: dict, *, flags: dict | None = None, device_memory: bool = False,
                 stream=None, kernel_ms=None, ldim: int = 0):
    """rrtmg_sw_run (radsw_main.F90:493) on the GPU; fills ``out`` in place.
    With ``device_memory`` every array (profile and outputs) must be a CUDA
    tensor (idxday and icseed included).  Raises on errflg."""
    keep = []
    a = make_run_args(prof, out, flags=flags, keep=keep, ldim=ldim)
    x = SwExec(precision=0, memory=1 if device_memory else 0, sync=1,
               stream=C.c_void_p(stream.cuda_stream if stream is not None else 0))
    km = None
    if kernel_ms is not None:
        km = (C.c_float * 3)()
        x.kernel_ms = C.cast(km, C.POINTER(C.c_float))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_sw_gpu_run_ex(C.byref(a), C.byref(x), msg, 512)
    if rc:
        raise RrtmgSwError(msg.value.decode())
    if km is not None:
        kernel_ms[:] = list(km)


def rrtmg_sw_run_blocks(profs, outs, *, flags: dict | None = None, ldims=None, stream=None, kernel_ms=None):
    """Many physics blocks in one rrtmg_sw_gpu_run_blocks call (device
    memory): profs[b] / outs[b] are block b's inputs and outputs (CUDA
    tensors), ldims[b] its leading dimension (0 = npts).  Same results as one
    rrtmg_sw_run per block.  Raises on errflg."""
    keep = []
    n = len(profs)
    arr = (SwRunArgs * max(n, 1))()
    for b in range(n):
        arr[b] = make_run_args(profs[b], outs[b], flags=flags, keep=keep, ldim=(ldims[b] if ldims else 0))
    x = SwExec(precision=0, memory=1, sync=1, stream=C.c_void_p(stream.cuda_stream if stream is not None else 0))
    km = None
    if kernel_ms is not None:
        km = (C.c_float * 3)()
        x.kernel_ms = C.cast(km, C.POINTER(C.c_float))
    msg = C.create_string_buffer(512)
    if lib().rrtmg_sw_gpu_run_blocks(arr, n, C.byref(x), msg, 512):
        raise RrtmgSwError(msg.value.decode())
    if km is not None:
        kernel_ms[:] = list(km)
