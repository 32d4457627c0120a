"""ctypes mirror of ``include/rrtmg_lw_gpu.h`` and helpers to fill it.

The argument struct carries the same names as the Fortran ``rrtmg_lw_run``
interface (physics/Radiation/RRTMG/radlw_main.F90:419-434) and ``rlwinit``
(radlw_main.F90:1322-1324).  Arrays are Fortran-ordered (column index
fastest): a profile field of shape ``(npts, nlay)`` in Fortran order is a
C-contiguous numpy/torch array of shape ``(nlay, npts)``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

NBANDS = 16
NGPT = 140

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

INPUT_FIELDS = (
    "plyr", "plvl", "tlyr", "tlvl", "qlyr", "olyr",
    "gasvmr_co2", "gasvmr_n2o", "gasvmr_ch4", "gasvmr_o2", "gasvmr_co",
    "gasvmr_cfc11", "gasvmr_cfc12", "gasvmr_cfc22", "gasvmr_ccl4",
)
OPTIONAL_CLOUD_FIELDS = (
    "cld_lwp", "cld_ref_liq", "cld_iwp", "cld_ref_ice", "cld_rwp",
    "cld_ref_rain", "cld_swp", "cld_ref_snow", "cld_od",
)
OUTPUT_FIELDS = ("hlwc", "topflx", "sfcflx", "cldtau")
OPTIONAL_OUTPUT_FIELDS = ("hlw0", "hlwb", "flxprf")


class InitArgs(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "me", "rad_hr_units", "inc_minor_gas", "ilwcliq", "isubclw", "iovr",
        "iovr_rand", "iovr_maxrand", "iovr_max", "iovr_dcorr", "iovr_exp",
        "iovr_exprand", "device")]


class RunArgs(C.Structure):
    _fields_ = (
        [(n, C.c_int32) for n in (
            "npts", "nlay", "nlp1", "ldim", "lprnt", "lslwr", "top_at_1",
            "inc_minor_gas", "iovr", "iovr_rand", "iovr_maxrand", "iovr_max",
            "iovr_dcorr", "iovr_exp", "iovr_exprand", "ilwcliq", "ilwcice",
            "isubclw")]
        + [(n, _dp) for n in INPUT_FIELDS]
        + [("icseed", _ip), ("aeraod", _dp), ("aerssa", _dp), ("sfemis", _dp),
           ("sfgtmp", _dp), ("dzlyr", _dp), ("delpin", _dp), ("de_lgth", _dp),
           ("alpha", _dp), ("cld_cf", _dp)]
        + [(n, _dp) for n in OPTIONAL_CLOUD_FIELDS]
        + [(n, _dp) for n in OUTPUT_FIELDS + OPTIONAL_OUTPUT_FIELDS]
    )


class ExecArgs(C.Structure):
    _fields_ = [("precision", C.c_int32), ("memory", C.c_int32),
                ("stream", C.c_void_p), ("sync", C.c_int32), ("reserved", C.c_int32),
                ("kernel_ms", C.POINTER(C.c_float))]


class Tuning(C.Structure):
    """rrtmg_lw_tuning: launch shape of the column kernels (0 = default)."""
    _fields_ = [("rt_warps", C.c_int32), ("gas_per_sm", C.c_int32), ("chunk_cols", C.c_int32),
                ("use_graph", C.c_int32)]


class SeedArgs(C.Structure):
    """rrtmg_lw_seed_args: seed part of GFS_rad_time_vary_timestep_init."""
    _fields_ = ([("sec", C.c_double)]
                + [(n, C.c_int32) for n in ("lslwr", "lsswr", "isubc_lw", "isubc_sw", "lrseeds", "ipsd0",
                                             "ipsdlim", "cnx", "cny", "isc", "jsc", "n", "ld_rseeds")]
                + [(n, _ip) for n in ("imap", "jmap", "rseeds", "icsdsw", "icsdlw")])


class OverlapArgs(C.Structure):
    """rrtmg_lw_overlap_args: decorrelation length and alpha (radiation_clouds.f:837-856)."""
    _fields_ = ([(n, C.c_int32) for n in ("mode", "npts", "nlay", "ldim", "idcor", "idcor_con", "idcor_hogan",
                                           "idcor_oreopoulos", "iovr", "iovr_dcorr", "iovr_exp",
                                           "iovr_exprand", "yearlen")]
                + [(n, C.c_double) for n in ("julian", "dcorr_con", "con_pi")]
                + [(n, _dp) for n in ("xlat", "latdeg", "dzlay", "cld_frac", "de_lgth", "alpha")])


class PostArgs(C.Structure):
    """rrtmg_lw_post_args: rrtmg_lw_post_run (rrtmg_lw_post.F90:13-77)."""
    _fields_ = ([(n, C.c_int32) for n in ("im", "levs", "ltp", "lm", "kd", "lslwr", "lwhtr")]
                + [(n, _dp) for n in ("tsfa", "htlwc", "htlw0", "sfcflw", "tsflw", "sfcdlw", "htrlw", "lwhc")])


OVERLAP_CLOUDS, OVERLAP_DCORR, OVERLAP_ALPHA = 0, 1, 2
# Decorrelation-length flags (radiation_clouds.f:447-450).
IDCOR_FLAGS = dict(idcor_con=0, idcor_hogan=1, idcor_oreopoulos=2)

FP64, FP32, SURROGATE = 0, 1, 2
HOST, DEVICE = 0, 1

# Standard GFS overlap flag values (GFS_typedefs / radiation_clouds).
OVERLAP_FLAGS = dict(iovr_rand=0, iovr_maxrand=1, iovr_max=2, iovr_dcorr=3,
                     iovr_exp=4, iovr_exprand=5)


def _check_dtype(name, x, kind):
    """Raise TypeError unless numpy array / torch tensor ``x`` holds ``kind``
    ("f8" for real(8), "i4" for int32); None passes."""
    if x is None:
        return
    want = {"f8": ("float64",), "i4": ("int32",)}[kind]
    got = str(x.dtype).replace("torch.", "")
    if got not in want:
        raise TypeError(f"{name} must be {want[0]}, got {got}")


def _ptr(x, ctype):
    """Pointer to the data of a numpy array or torch tensor (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be contiguous")
        return x.ctypes.data_as(C.POINTER(ctype))
    # torch tensor (host or device)
    if not x.is_contiguous():
        raise ValueError("tensors must be contiguous")
    return C.cast(C.c_void_p(x.data_ptr()), C.POINTER(ctype))


def make_init_args(rad_hr_units=1, inc_minor_gas=True, ilwcliq=1, isubclw=2,
                   iovr=1, me=1, device=0, **overlap):
    flags = dict(OVERLAP_FLAGS)
    flags.update(overlap)
    return InitArgs(me=me, rad_hr_units=rad_hr_units, inc_minor_gas=int(inc_minor_gas),
                    ilwcliq=ilwcliq, isubclw=isubclw, iovr=iovr, device=device, **flags)


def make_run_args(prof: dict, out: dict, *, flags: dict | None = None, keep=None) -> RunArgs:
    """Fill a RunArgs from a profile dict (see ``synthetic.make_profiles``) and
    an output dict.  ``keep`` (a list) receives the objects whose memory the
    struct points at, so the caller can hold them alive."""
    f = dict(prof["flags"])
    if flags:
        f.update(flags)
    npts, nlay = prof["npts"], prof["nlay"]
    a = RunArgs()
    a.npts, a.nlay, a.nlp1 = npts, nlay, nlay + 1
    a.ldim = f.get("ldim", 0)
    for n in ("lprnt", "lslwr", "top_at_1", "inc_minor_gas", "iovr", "ilwcliq",
              "ilwcice", "isubclw"):
        setattr(a, n, int(f[n]))
    for n, v in OVERLAP_FLAGS.items():
        setattr(a, n, int(f.get(n, v)))
    for n in INPUT_FIELDS + ("aeraod", "aerssa", "sfemis", "sfgtmp", "dzlyr", "delpin",
                             "de_lgth", "alpha", "cld_cf") + OPTIONAL_CLOUD_FIELDS:
        setattr(a, n, _ptr(prof.get(n), C.c_double))
    a.icseed = _ptr(prof.get("icseed"), C.c_int32)
    for n in OUTPUT_FIELDS + OPTIONAL_OUTPUT_FIELDS:
        setattr(a, n, _ptr(out.get(n), C.c_double))
    if keep is not None:
        keep.extend([prof, out])
    return a


def alloc_outputs(npts, nlay, *, hlw0=True, hlwb=False, flxprf=False, like=None):
    """Output arrays in Fortran order, filled with NaN so unwritten values show."""
    def mk(shape):
        if like is None:
            return np.full(shape, np.nan)
        import torch
        return torch.full(shape, float("nan"), dtype=torch.float64, device=like)
    out = {"hlwc": mk((nlay, npts)), "topflx": mk((npts, 2)), "sfcflx": mk((npts, 4)),
           "cldtau": mk((nlay, npts))}
    if hlw0:
        out["hlw0"] = mk((nlay, npts))
    if hlwb:
        out["hlwb"] = mk((NBANDS, nlay, npts))
    if flxprf:
        out["flxprf"] = mk((nlay + 1, npts, 4))
    return out
