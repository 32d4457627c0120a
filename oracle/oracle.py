"""ctypes front end of the CPU restatement of the RRTMG-LW path.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline / reference arm, never by the product package.
The restatement itself is ``rrtmg_lw_oracle.cpp`` (see its header for the
reference lines it follows and for the parity-pinning status).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from ccpp_physics_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librrtmg_lw_oracle.so")
TABLES = os.path.join(HERE, "..", "ccpp_physics_b200", "data", "rrtmg_lw_tables.bin")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.oracle_rlwinit.argtypes = [C.c_char_p, C.POINTER(abi.InitArgs), C.c_char_p, C.c_int]
        L.oracle_rrtmg_lw_run.argtypes = [C.POINTER(abi.RunArgs), C.c_int, C.c_char_p, C.c_int]
        L.oracle_column_stages.argtypes = [C.POINTER(abi.RunArgs), C.c_int, C.c_void_p] + \
            [C.c_void_p] * 9 + [C.c_char_p, C.c_int]
        L.oracle_mt_stream.argtypes = [C.c_int32, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_mcica.argtypes = [C.c_int, C.c_int32, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_double, C.c_void_p, C.c_void_p]
        L.oracle_tables.argtypes = [C.c_void_p] * 4
        L.oracle_check_u32_unit.argtypes = [C.c_ulonglong, C.c_ulonglong]
        L.oracle_check_u32_unit.restype = C.c_ulonglong
        _lib = L
    return _lib


def _vp(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def rlwinit(rad_hr_units=1, iovr=1, **kw):
    ia = abi.make_init_args(rad_hr_units=rad_hr_units, iovr=iovr, **kw)
    msg = C.create_string_buffer(512)
    rc = lib().oracle_rlwinit(TABLES.encode(), C.byref(ia), msg, 512)
    return rc, msg.value.decode()


def rrtmg_lw_run(prof, *, hlw0=True, hlwb=False, flxprf=False, nthreads=0, flags=None, out=None):
    """Run the oracle on a numpy profile dict; returns (errflg, errmsg, out)."""
    npts, nlay = prof["npts"], prof["nlay"]
    if out is None:
        out = abi.alloc_outputs(npts, nlay, hlw0=hlw0, hlwb=hlwb, flxprf=flxprf)
    keep = []
    a = abi.make_run_args(prof, out, flags=flags, keep=keep)
    msg = C.create_string_buffer(512)
    rc = lib().oracle_rrtmg_lw_run(C.byref(a), nthreads, msg, 512)
    return rc, msg.value.decode(), out


def column_stages(prof, icol, flags=None):
    """Per-stage internals of column ``icol`` (0-based); Fortran layouts."""
    nlay = prof["nlay"]
    keep = []
    out = abi.alloc_outputs(prof["npts"], nlay)
    a = abi.make_run_args(prof, out, flags=flags, keep=keep)
    ints = np.zeros(1 + 3 * nlay, dtype=np.int32)
    r = {n: np.zeros((nlay, 140)) for n in ("taug", "fracs", "tautot", "cldfmc")}
    r["taucld"] = np.zeros((nlay, 16))
    r["pklay"] = np.zeros((nlay + 1, 16))
    r["pklev"] = np.zeros((nlay + 1, 16))
    sc = np.zeros(17)
    fac = np.zeros(13 * nlay)
    msg = C.create_string_buffer(512)
    rc = lib().oracle_column_stages(C.byref(a), icol + 1, _vp(ints), _vp(r["taug"]), _vp(r["fracs"]),
                                    _vp(r["tautot"]), _vp(r["cldfmc"]), _vp(r["taucld"]),
                                    _vp(r["pklay"]), _vp(r["pklev"]), _vp(sc), _vp(fac), msg, 512)
    if rc:
        raise RuntimeError(msg.value.decode())
    r["laytrop"] = int(ints[0])
    r["jp"], r["jt"], r["jt1"] = ints[1:1 + nlay], ints[1 + nlay:1 + 2 * nlay], ints[1 + 2 * nlay:]
    r["pwvcm"], r["secdiff"] = sc[0], sc[1:]
    f = fac.reshape(13, nlay)
    r["fac00"], r["fac01"], r["fac10"], r["fac11"] = f[0], f[1], f[2], f[3]
    r["colamt"] = f[4:11]
    r["coldry"], r["colbrd"] = f[11], f[12]
    return r


def mt_stream(seed, n):
    u = np.zeros(n, dtype=np.uint32)
    x = np.zeros(n)
    st = np.zeros(624, dtype=np.uint32)
    lib().oracle_mt_stream(seed, n, _vp(u), _vp(x), _vp(st))
    return u, x, st


def mcica(cldf, seed, iovr=1, dz=None, de_lgth=2.0, alpha=None):
    cldf = np.ascontiguousarray(cldf, dtype=np.float64)
    nlay = cldf.size
    out = np.zeros((nlay, 140), dtype=np.uint8)
    dz = None if dz is None else np.ascontiguousarray(dz, dtype=np.float64)
    alpha = None if alpha is None else np.ascontiguousarray(alpha, dtype=np.float64)
    lib().oracle_mcica(nlay, seed, iovr, _vp(cldf), _vp(dz), de_lgth, _vp(alpha), _vp(out))
    return out.astype(bool)


def tables():
    tau = np.zeros(10001)
    ex = np.zeros(10001)
    tfn = np.zeros(10001)
    fh = np.zeros(2)
    lib().oracle_tables(_vp(tau), _vp(ex), _vp(tfn), _vp(fh))
    return tau, ex, tfn, fh
