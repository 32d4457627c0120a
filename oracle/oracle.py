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
        L.oracle_random_index.argtypes = [C.c_int32, C.c_int32, C.c_longlong, C.c_void_p]
        L.oracle_seeds.argtypes = [C.c_double] + [C.c_int32] * 13 + [C.c_void_p] * 5
        L.oracle_dcorr_hogan.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p]
        L.oracle_dcorr_oreopoulos.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_void_p]
        L.oracle_alpha_exper.argtypes = [C.c_int] * 5 + [C.c_void_p] * 4
        L.oracle_overlap_params.argtypes = ([C.c_int] * 7 + [C.c_double, C.c_void_p, C.c_void_p, C.c_double,
                                            C.c_int, C.c_double] + [C.c_int] * 4 + [C.c_void_p] * 4)
        L.oracle_post.argtypes = [C.c_int] * 7 + [C.c_void_p] * 8
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


# ---- steps either side of rrtmg_lw_run ----------------------------------------

def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def random_index(seed, imax, m):
    """random_setseed_t(seed) then random_index_t(imax, out(m))."""
    out = np.zeros(m, dtype=np.int32)
    lib().oracle_random_index(seed, imax, m, _vp(out))
    return out


def seeds(*, sec, ipsd0, ipsdlim, cnx, cny, isc, jsc, imap, jmap, lslwr=1, lsswr=1, isubc_lw=2, isubc_sw=2,
          lrseeds=0, rseeds=None, icsdsw=None, icsdlw=None):
    """Seed part of GFS_rad_time_vary_timestep_init; returns (rc, icsdsw, icsdlw).
    ``rseeds`` is the (n, 2) Fortran array as a C-contiguous (2, n) array."""
    imap = np.ascontiguousarray(imap, dtype=np.int32)
    jmap = np.ascontiguousarray(jmap, dtype=np.int32)
    n = imap.size
    sw = np.zeros(n, dtype=np.int32) if icsdsw is None else icsdsw
    lw = np.zeros(n, dtype=np.int32) if icsdlw is None else icsdlw
    rs = None if rseeds is None else np.ascontiguousarray(rseeds, dtype=np.int32)
    ld = 0 if rs is None else rs.shape[-1]
    rc = lib().oracle_seeds(float(sec), lslwr, lsswr, isubc_lw, isubc_sw, lrseeds, ipsd0, ipsdlim, cnx, cny, isc,
                            jsc, n, ld, _vp(imap), _vp(jmap), _vp(rs), _vp(sw), _vp(lw))
    return rc, sw, lw


def dcorr_hogan(lat, con_pi=np.pi):
    lat = _f64(lat)
    out = np.zeros_like(lat)
    lib().oracle_dcorr_hogan(lat.size, _vp(lat), con_pi, _vp(out))
    return out


def dcorr_oreopoulos(lat, juldat, yearlength):
    lat = _f64(lat)
    out = np.zeros_like(lat)
    lib().oracle_dcorr_oreopoulos(lat.size, _vp(lat), float(juldat), int(yearlength), _vp(out))
    return out


def alpha_exper(iovr, iovr_exprand, dzlay, dcorr, cld_frac):
    """(nlay, ncol) C-contiguous = Fortran (ncol, nlay)."""
    dzlay, dcorr, cld_frac = _f64(dzlay), _f64(dcorr), _f64(cld_frac)
    nlay, ncol = dzlay.shape
    out = np.zeros_like(dzlay)
    lib().oracle_alpha_exper(ncol, nlay, ncol, iovr, iovr_exprand, _vp(dzlay), _vp(dcorr), _vp(cld_frac), _vp(out))
    return out


def overlap_params(iovr, idcor, dzlay, cld_frac, *, xlat=None, latdeg=None, julian=0.0, yearlen=365,
                   dcorr_con=2.5, con_pi=np.pi, de_lgth=None, idcor_flags=(0, 1, 2), iovr_flags=(3, 4, 5)):
    """radiation_clouds.f:837-856; returns (de_lgth, alpha)."""
    dzlay, cld_frac = _f64(dzlay), _f64(cld_frac)
    nlay, ncol = dzlay.shape
    dl = np.zeros(ncol) if de_lgth is None else _f64(de_lgth).copy()
    al = np.zeros_like(dzlay)
    c, h, o = idcor_flags
    lib().oracle_overlap_params(ncol, nlay, ncol, idcor, c, h, o, float(dcorr_con), _vp(_f64(xlat)),
                                _vp(_f64(latdeg)), float(julian), int(yearlen), float(con_pi), iovr, *iovr_flags,
                                _vp(dzlay), _vp(cld_frac), _vp(dl), _vp(al))
    return dl, al


def post(im, levs, ltp, lm, kd, lslwr, lwhtr, tsfa, htlwc, htlw0, sfcflw, tsflw, sfcdlw, htrlw, lwhc):
    """rrtmg_lw_post_run on numpy arrays (outputs in place)."""
    lib().oracle_post(im, levs, ltp, lm, kd, int(lslwr), int(lwhtr), _vp(tsfa), _vp(htlwc), _vp(htlw0),
                      _vp(sfcflw), _vp(tsflw), _vp(sfcdlw), _vp(htrlw), _vp(lwhc))
