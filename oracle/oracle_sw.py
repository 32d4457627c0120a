"""ctypes front end of the CPU restatement of the RRTMG-SW path.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline / reference arm, never by the product package.
The restatement itself is ``rrtmg_sw_oracle.cpp`` (see its header for the
reference lines it follows and for the parity-pinning status).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from ccpp_physics_b200 import rrtmg_sw as sw

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librrtmg_sw_oracle.so")
TABLES = os.path.join(HERE, "..", "ccpp_physics_b200", "data", "rrtmg_sw_tables.bin")

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE, "librrtmg_sw_oracle.so"], check=True)
        L = C.CDLL(LIB_PATH)
        L.oracle_rswinit.argtypes = [C.c_char_p, C.POINTER(sw.SwInitArgs), C.c_char_p, C.c_int]
        L.oracle_rrtmg_sw_run.argtypes = [C.POINTER(sw.SwRunArgs), C.c_int, C.c_char_p, C.c_int]
        L.oracle_sw_gas_optics.argtypes = [C.POINTER(sw.SwRunArgs), C.c_int] + [C.c_void_p] * 3
        L.oracle_sw_mcica.argtypes = [C.c_int, C.c_int32, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                      C.c_void_p, C.c_void_p]
        L.oracle_sw_pre.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_int32), C.c_void_p]
        L.oracle_sw_pre.restype = None
        L.oracle_sw_post.argtypes = [C.POINTER(sw.SwPostArgs)]
        L.oracle_sw_post.restype = None
        _lib = L
    return _lib


def rswinit(rad_hr_units=1, iovr=1, iswmode=2, iswcliq=1, isubcsw=2):
    a = sw.make_init_args(rad_hr_units=rad_hr_units, iovr=iovr, iswmode=iswmode, iswcliq=iswcliq,
                          isubcsw=isubcsw)
    msg = C.create_string_buffer(256)
    rc = lib().oracle_rswinit(TABLES.encode(), C.byref(a), msg, 256)
    return rc, msg.value.decode()


def run(prof, out, flags=None, nthreads=0, ldim=0):
    """rrtmg_sw_run on the CPU; fills ``out`` (numpy) in place.  Returns
    (errflg, errmsg)."""
    keep = []
    a = sw.make_run_args(prof, out, flags=flags, keep=keep, ldim=ldim)
    msg = C.create_string_buffer(512)
    rc = lib().oracle_rrtmg_sw_run(C.byref(a), nthreads, msg, 512)
    return rc, msg.value.decode()


def gas_optics(prof, ipt, flags=None):
    """taug, taur (nlay, 112) in internal order, sfluxzen (112,), laytrop of
    daytime point ipt (1-based)."""
    keep = []
    out = sw.alloc_outputs(prof["npts"], prof["nlay"])
    a = sw.make_run_args(prof, out, flags=flags, keep=keep)
    nl = prof["nlay"]
    taug, taur, sf = np.zeros((nl, sw.NGPT)), np.zeros((nl, sw.NGPT)), np.zeros(sw.NGPT)
    lt = lib().oracle_sw_gas_optics(C.byref(a), ipt, taug.ctypes.data_as(C.c_void_p),
                                    taur.ctypes.data_as(C.c_void_p), sf.ctypes.data_as(C.c_void_p))
    return taug, taur, sf, lt


def mcica_bits(nlay, seed, iovr, cldf, dz=None, de_lgth=0.0, alpha=None):
    nw = (nlay + 31) // 32
    bits = np.zeros((sw.NGPT, nw), np.uint32)
    vp = lambda x: None if x is None else np.ascontiguousarray(x, np.float64).ctypes.data_as(C.c_void_p)
    cl = np.ascontiguousarray(cldf, np.float64)
    lib().oracle_sw_mcica(nlay, seed, iovr, cl.ctypes.data_as(C.c_void_p), vp(dz), de_lgth, vp(alpha),
                          bits.ctypes.data_as(C.c_void_p))
    return bits


def post(im, levr, levs, ltp, nday, lm, kd, lsswr, swhtr, sfcalb1, sfcalb2, sfcalb3, sfcalb4, htswc, htsw0,
         nirbmdi, nirdfdi, visbmdi, visdfdi, nirbmui, nirdfui, visbmui, visdfui, sfcdsw, sfcnsw, htrsw, swhc,
         scmpsw, sfcfsw, topfsw):
    """rrtmg_sw_post_run on numpy arrays (outputs and records in place), the
    argument order of ``ccpp_physics_b200.rrtmg_sw_post.rrtmg_sw_post_run``."""
    vals = locals()
    a = sw.SwPostArgs(im=im, levr=levr, levs=levs, ltp=ltp, nday=nday, lm=lm, kd=kd, lsswr=int(bool(lsswr)),
                      swhtr=int(bool(swhtr)))
    for n in sw.POST_INPUT_FIELDS + sw.POST_OUTPUT_FIELDS:
        v = vals[n]
        if v is not None:
            assert v.dtype == np.float64 and v.flags["C_CONTIGUOUS"], n
            setattr(a, n, v.ctypes.data_as(C.POINTER(C.c_double)))
    lib().oracle_sw_post(C.byref(a))


def pre(im, lsswr, coszen):
    """rad_sw_pre_run: returns (nday, idxday (im,) int32)."""
    idx = np.zeros(im, np.int32)
    nday = C.c_int32(0)
    cz = np.ascontiguousarray(coszen, np.float64)
    lib().oracle_sw_pre(im, int(bool(lsswr)), cz.ctypes.data_as(C.c_void_p), C.byref(nday),
                        idx.ctypes.data_as(C.c_void_p))
    return nday.value, idx
