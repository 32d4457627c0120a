"""Seeded synthetic atmospheric profiles for the RRTMG-LW column path.

The reference publishes no dataset for this path, so every workload is a
seeded synthetic stand-in with the shapes and value distributions below.
Each random draw is a counter-based hash of (seed, column, field, layer),
so a column's profile depends only on its global index: the same column is
identical whatever physics-block partitioning or chunking produced it, and
the generator runs vectorised on the CPU or directly on the GPU (torch).

Profile model (per column):
* levels: reference pressures log-uniform from 1000 hPa (surface) to
  0.2 hPa, hybrid sigma-pressure B = max(0, (p_r-100)/900)**1.5,
  p = p_r (1-B) + B ps with ps ~ U(950, 1030) hPa; plyr = level mean,
  delpin = level difference, dzlyr hypsometric [km];
* temperature: Tsfc ~ U(250, 305) K, -6.5 K/km up to a tropopause at
  p_trop ~ U(100, 250) hPa, then +1 K/km, plus N(0, 2 K) per layer; level
  temperatures interpolated in ln p, surface level = Tsfc;
* H2O: relative humidity U(0.1, 0.95) per layer below the tropopause
  (Magnus saturation), 3 ppmv above; passed as specific humidity;
* O3: 8 ppmv * exp(-(ln p - ln 10)^2 / (2 0.8^2)), passed as mass mixing
  ratio; CO2 400, CH4 1.8, N2O 0.32 ppmv, O2 0.209, CO 1.5e-8, CFC-11/12/22
  and CCl4 at the default vmr of physics/Radiation/radiation_gases.f:145-153;
* surface: emissivity U(0.95, 1), ground temperature = lowest layer T +
  U(-5, 5) K; aerosol optical depth and single-scattering albedo zero;
* clouds (all-sky configs): cf = clip((RH-0.8)/0.2, 0, 1); where cf > 0 a
  liquid path LogN(ln 20 g/m2, 1) if T > 253 K else an ice path
  LogN(ln 10 g/m2, 1.2); re_liq ~ U(5, 15) um, re_ice ~ U(20, 80) um; no
  rain or snow; decorrelation length 2 km;
* McICA seed of column i = its global index (seed 0 becomes 4357 inside
  the Mersenne twister, mersenne_twister.f:291).
"""
from __future__ import annotations

import math

import numpy as np
import torch

CON_G = 9.80665
CON_AMD = 28.9644
CON_AMW = 18.0154
CON_AMO3 = 47.9982
RD = 287.05

GASES = dict(gasvmr_co2=400e-6, gasvmr_n2o=0.32e-6, gasvmr_ch4=1.8e-6, gasvmr_o2=0.209,
             gasvmr_co=1.5e-8, gasvmr_cfc11=3.52e-10, gasvmr_cfc12=6.358e-10,
             gasvmr_cfc22=1.5e-10, gasvmr_ccl4=1.397e-10)

DEFAULT_FLAGS = dict(lprnt=0, lslwr=1, top_at_1=0, inc_minor_gas=1, iovr=1, ilwcliq=1,
                     ilwcice=3, isubclw=2)

_M32 = 0xFFFFFFFF


def _mul32(x, c):
    """(x * c) mod 2**32 for 0 <= x < 2**32 without int64 overflow."""
    lo, hi = c & 0xFFFF, c >> 16
    return ((x * lo) + (((x * hi) & 0xFFFF) << 16)) & _M32


def _mix32(x):
    x = x ^ (x >> 16)
    x = _mul32(x, 0x7FEB352D)
    x = x ^ (x >> 15)
    x = _mul32(x, 0x846CA68B)
    return x ^ (x >> 16)


def _uniform(seed, col, field, layer=None):
    """U(0,1) as float64, shape broadcast of col (1, n) and layer (L, 1)."""
    h = _mix32(torch.full_like(col, (seed & _M32)) ^ ((field * 0x9E3779B1) & _M32))
    h = _mix32(h ^ (col & _M32))
    if layer is not None:
        h = _mix32(h ^ (((layer + 1) * 0x85EBCA77) & _M32))
    return (h.to(torch.float64) + 0.5) * (1.0 / 4294967296.0)


def _normal(seed, col, field, layer=None):
    u1 = _uniform(seed, col, field, layer)
    u2 = _uniform(seed, col, field + 1000, layer)
    return torch.sqrt(-2.0 * torch.log(u1)) * torch.cos(2.0 * math.pi * u2)


def make_profiles(npts: int, nlay: int, *, seed: int = 1, col_offset: int = 0,
                  cloudy: bool = True, device="cpu", as_numpy: bool | None = None):
    """Generate ``npts`` columns x ``nlay`` layers.  Fields are Fortran-ordered:
    (npts, nlay) arrays are returned as C-contiguous (nlay, npts), aerosols as
    (16, nlay, npts).  Returns a dict with the fields, ``npts``, ``nlay`` and
    the default ``flags``."""
    dev = torch.device(device)
    if as_numpy is None:
        as_numpy = dev.type == "cpu"
    f64 = dict(dtype=torch.float64, device=dev)
    col = (torch.arange(npts, dtype=torch.int64, device=dev) + col_offset).reshape(1, npts)
    lay = torch.arange(nlay, dtype=torch.int64, device=dev).reshape(nlay, 1)
    lev = torch.arange(nlay + 1, dtype=torch.int64, device=dev).reshape(nlay + 1, 1)

    ps = 950.0 + 80.0 * _uniform(seed, col, 1)
    tsfc = 250.0 + 55.0 * _uniform(seed, col, 2)
    ptrop = 100.0 + 150.0 * _uniform(seed, col, 3)

    pr = torch.exp(torch.linspace(math.log(1000.0), math.log(0.2), nlay + 1, **f64)).reshape(-1, 1)
    bk = torch.clamp((pr - 100.0) / 900.0, min=0.0) ** 1.5
    plvl = pr * (1.0 - bk) + bk * ps
    plvl[0] = ps[0]
    plvl[-1] = 0.2
    plyr = 0.5 * (plvl[:-1] + plvl[1:])
    delp = plvl[:-1] - plvl[1:]

    # level temperatures by hypsometric integration of the lapse-rate model
    tlev = torch.empty((nlay + 1, npts), **f64)
    z = torch.zeros((1, npts), **f64)
    ztrop = torch.full((1, npts), float("inf"), **f64)
    for k in range(nlay + 1):
        above = plvl[k:k + 1] <= ptrop
        ztrop = torch.where(above & torch.isinf(ztrop), z, ztrop)
        ttrop = tsfc - 6.5 * ztrop
        t = torch.where(above, ttrop + 1.0 * (z - ztrop), tsfc - 6.5 * z)
        tlev[k] = t[0]
        if k < nlay:
            z = z + (RD * t / CON_G) * torch.log(plvl[k:k + 1] / plvl[k + 1:k + 2]) / 1000.0
    tlyr = 0.5 * (tlev[:-1] + tlev[1:]) + 2.0 * _normal(seed, col, 10, lay)
    lnpl, lnpv = torch.log(plyr), torch.log(plvl)
    tlvl = torch.empty_like(tlev)
    tlvl[0] = tsfc[0]
    w = (lnpv[1:nlay] - lnpl[:-1]) / (lnpl[1:] - lnpl[:-1])
    tlvl[1:nlay] = tlyr[:-1] + w * (tlyr[1:] - tlyr[:-1])
    tlvl[nlay] = tlyr[nlay - 1]
    dz = (RD * tlyr / CON_G) * torch.log(plvl[:-1] / plvl[1:]) / 1000.0

    trop = plyr > ptrop
    rh = 0.1 + 0.85 * _uniform(seed, col, 20, lay)
    es = 6.1094 * torch.exp(17.625 * (tlyr - 273.15) / (tlyr - 30.11))
    es = torch.minimum(es, 0.5 * plyr)
    qs = 0.622 * es / (plyr - 0.378 * es)
    amdw = CON_AMD / CON_AMW
    q_strat = 3e-6 / (amdw + 3e-6)
    q = torch.where(trop, rh * qs, torch.full_like(qs, q_strat))
    o3vmr = 8e-6 * torch.exp(-(lnpl - math.log(10.0)) ** 2 / (2.0 * 0.8 ** 2))
    olyr = o3vmr * CON_AMO3 / CON_AMD

    prof = dict(npts=npts, nlay=nlay, flags=dict(DEFAULT_FLAGS))
    prof.update(plyr=plyr, plvl=plvl, tlyr=tlyr, tlvl=tlvl, qlyr=q, olyr=olyr,
                dzlyr=dz, delpin=delp)
    for name, v in GASES.items():
        prof[name] = torch.full((nlay, npts), v, **f64)
    prof["sfemis"] = (0.95 + 0.05 * _uniform(seed, col, 30))[0]
    prof["sfgtmp"] = (tlyr[0:1] - 5.0 + 10.0 * _uniform(seed, col, 31))[0]
    prof["aeraod"] = torch.zeros((16, nlay, npts), **f64)
    prof["aerssa"] = torch.zeros((16, nlay, npts), **f64)
    prof["icseed"] = (col[0] & 0x7FFFFFFF).to(torch.int32)
    prof["de_lgth"] = torch.full((npts,), 2.0, **f64)
    dzm = torch.cat([dz[:1], 0.5 * (dz[1:] + dz[:-1])], dim=0)
    prof["alpha"] = torch.exp(-dzm / 2.0)
    if cloudy:
        cf = torch.where(trop, torch.clamp((rh - 0.8) / 0.2, 0.0, 1.0), torch.zeros_like(rh))
        has = cf > 0.0
        warm = tlyr > 253.0
        lwp = torch.exp(math.log(20.0) + 1.0 * _normal(seed, col, 40, lay))
        iwp = torch.exp(math.log(10.0) + 1.2 * _normal(seed, col, 42, lay))
        prof["cld_cf"] = cf
        prof["cld_lwp"] = torch.where(has & warm, lwp, torch.zeros_like(lwp))
        prof["cld_iwp"] = torch.where(has & ~warm, iwp, torch.zeros_like(iwp))
        prof["cld_ref_liq"] = 5.0 + 10.0 * _uniform(seed, col, 44, lay)
        prof["cld_ref_ice"] = 20.0 + 60.0 * _uniform(seed, col, 45, lay)
    else:
        prof["cld_cf"] = torch.zeros((nlay, npts), **f64)
        prof["cld_lwp"] = torch.zeros((nlay, npts), **f64)
        prof["cld_iwp"] = torch.zeros((nlay, npts), **f64)
        prof["cld_ref_liq"] = torch.full((nlay, npts), 10.0, **f64)
        prof["cld_ref_ice"] = torch.full((nlay, npts), 50.0, **f64)
    for n in ("cld_rwp", "cld_ref_rain", "cld_swp", "cld_ref_snow"):
        prof[n] = torch.zeros((nlay, npts), **f64)
    if as_numpy:
        for k, v in list(prof.items()):
            if isinstance(v, torch.Tensor):
                prof[k] = np.ascontiguousarray(v.cpu().numpy())
    else:
        for k, v in list(prof.items()):
            if isinstance(v, torch.Tensor):
                prof[k] = v.contiguous()
    return prof


def physics_blocks(total: int, seed: int = 7, lo: int = 8, hi: int = 256):
    """Uneven UFS-style physics block sizes, U{lo..hi}, summing to ``total``
    (the last block truncated)."""
    rng = np.random.default_rng(seed)
    sizes = []
    s = 0
    while s < total:
        b = int(rng.integers(lo, hi + 1))
        b = min(b, total - s)
        sizes.append(b)
        s += b
    return np.asarray(sizes, dtype=np.int32)


def slice_columns(prof: dict, start: int, stop: int) -> dict:
    """Columns [start, stop) of a profile dict (copies, Fortran layout kept)."""
    out = dict(npts=stop - start, nlay=prof["nlay"], flags=dict(prof["flags"]))
    for k, v in prof.items():
        if k in ("npts", "nlay", "flags"):
            continue
        sub = v[..., start:stop]
        out[k] = np.ascontiguousarray(sub) if isinstance(v, np.ndarray) else sub.contiguous()
    return out
