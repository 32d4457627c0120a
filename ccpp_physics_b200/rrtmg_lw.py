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


def run_profile(prof: dict, out: dict, *, precision="fp64", flags=None, stream=None, sync=True):
    """rrtmg_lw_run over a profile dict (field name -> array) into ``out``.
    Returns (errmsg, errflg) like the Fortran routine."""
    keep = []
    a = abi.make_run_args(prof, out, flags=flags, keep=keep)
    device = _is_device(prof["plyr"])
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


def mcica_bits(cldf, seed, iovr=1, stream=None):
    """Sub-column cloud flags of ``mcica_subcol`` on the GPU for device
    tensors cldf (nlay, npts) float64 and seed (npts,) int32.  Returns a
    (npts, 140, nwords) int32 tensor of bit words (bit k&31 of word k>>5)."""
    import torch
    nlay, npts = cldf.shape
    nw = (nlay + 31) // 32
    bits = torch.zeros((npts, abi.NGPT, nw), dtype=torch.int32, device=cldf.device)
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_mcica(npts, nlay, npts, iovr, C.c_void_p(seed.data_ptr()),
                                  C.c_void_p(cldf.data_ptr()), None, None, None,
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
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_gas_optics(C.byref(a), PRECISIONS[precision], C.c_void_p(taug.data_ptr()),
                                       C.c_void_p(fracs.data_ptr()), stream, msg, 512)
    if rc:
        raise RRTMGLWError(msg.value.decode())
    return taug, fracs


def to_device(prof: dict, device="cuda"):
    """Copy a numpy profile dict to device tensors (Fortran layout kept)."""
    import torch
    out = dict(npts=prof["npts"], nlay=prof["nlay"], flags=dict(prof["flags"]))
    for k, v in prof.items():
        if isinstance(v, np.ndarray):
            out[k] = torch.from_numpy(v).to(device)
    return out
