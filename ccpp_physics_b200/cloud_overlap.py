"""Cloud-overlap parameters on the GPU: ``module_radiation_cloud_overlap``
(physics/Radiation/radiation_cloud_overlap.F90) and the block of
radiation_clouds.f:837-856 that calls it.

* ``cmp_dcorr_lgth_hogan`` (:28-50) and ``cmp_dcorr_lgth_oreopoulos`` (:58-93):
  the decorrelation length ``de_lgth`` (km) per column;
* ``get_alpha_exper`` (:99-145): the overlap parameter alpha per layer for the
  exponential overlaps;
* ``overlap_params``: the radiation_clouds.f block (de_lgth by ``idcor``, then
  alpha for iovr dcorr/exp/exprand, both zero otherwise) -- the ``de_lgth``
  and ``alpha`` that ``rrtmg_lw_run`` takes.

Arrays are Fortran-ordered ``(npts[, nlay])`` fields: numpy (host) or torch
CUDA tensors (device), float64; outputs are filled in place and each call
returns ``(errmsg, errflg)``.  Runs in ``librrtmg_lw_gpu.so``
(``rrtmg_lw_gpu_overlap_params``).
"""
from __future__ import annotations

import ctypes as C
import math

from . import abi
from .rrtmg_lw import _is_device, lib, torch_stream


def _IOVR(flags):
    """The exponential-overlap codes (the only iovr codes these steps read)."""
    return {n: int(flags[n]) for n in ("iovr_dcorr", "iovr_exp", "iovr_exprand")}


def _call(a, ref, stream, sync):
    st = torch_stream(stream, ref)
    x = abi.ExecArgs(memory=abi.DEVICE if _is_device(ref) else abi.HOST,
                     stream=None if st is None else C.c_void_p(st), sync=int(sync))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_overlap_params(C.byref(a), C.byref(x), msg, 512)
    return msg.value.decode(), rc


def _args(mode, npts, nlay, **kw):
    ptrs = {n: abi._ptr(kw.pop(n, None), C.c_double) for n in ("xlat", "latdeg", "dzlay", "cld_frac",
                                                                "de_lgth", "alpha")}
    a = abi.OverlapArgs(mode=mode, npts=npts, nlay=nlay, ldim=0, **abi.IDCOR_FLAGS, **_IOVR(abi.OVERLAP_FLAGS))
    for n, v in kw.items():
        setattr(a, n, v)
    for n, v in ptrs.items():
        setattr(a, n, v)
    return a


def cmp_dcorr_lgth_hogan(lat, con_pi, dcorr_lgth, *, stream=None, sync=True):
    """Hogan et al. (2010) eq. 13; lat in radians."""
    a = _args(abi.OVERLAP_DCORR, int(lat.shape[-1]), 0, idcor=abi.IDCOR_FLAGS["idcor_hogan"],
              con_pi=float(con_pi), xlat=lat, de_lgth=dcorr_lgth)
    return _call(a, dcorr_lgth, stream, sync)


def cmp_dcorr_lgth_oreopoulos(lat, juldat, yearlength, dcorr_lgth, *, stream=None, sync=True):
    """Oreopoulos et al. (2012) eqs. 10-11; lat in degrees."""
    a = _args(abi.OVERLAP_DCORR, int(lat.shape[-1]), 0, idcor=abi.IDCOR_FLAGS["idcor_oreopoulos"],
              julian=float(juldat), yearlen=int(yearlength), latdeg=lat, de_lgth=dcorr_lgth)
    return _call(a, dcorr_lgth, stream, sync)


def get_alpha_exper(iovr, iovr_exprand, dzlay, dcorr_lgth, cld_frac, alpha, *, stream=None, sync=True):
    """alpha(:,1) = 0, alpha(:,k) = exp(-dzlay(:,k) / dcorr_lgth); for
    iovr == iovr_exprand, 0 where a clear layer follows a cloudy one."""
    nlay, npts = alpha.shape
    a = _args(abi.OVERLAP_ALPHA, npts, nlay, iovr=int(iovr), iovr_exprand=int(iovr_exprand), dzlay=dzlay,
              cld_frac=cld_frac, de_lgth=dcorr_lgth, alpha=alpha)
    return _call(a, alpha, stream, sync)


def overlap_params(iovr, idcor, dzlay, cld_frac, de_lgth, alpha, *, xlat=None, latdeg=None, julian=0.0,
                   yearlen=365, dcorr_con=2.5, con_pi=math.pi, idcor_flags=None, iovr_flags=None,
                   stream=None, sync=True):
    """The radiation_clouds.f:837-856 block; flag codes default to the GFS ones."""
    nlay, npts = alpha.shape
    flags = dict(abi.IDCOR_FLAGS, **(idcor_flags or {}))
    flags.update(_IOVR(dict(abi.OVERLAP_FLAGS, **(iovr_flags or {}))))
    a = _args(abi.OVERLAP_CLOUDS, npts, nlay, idcor=int(idcor), iovr=int(iovr), julian=float(julian),
              yearlen=int(yearlen), dcorr_con=float(dcorr_con), con_pi=float(con_pi), xlat=xlat, latdeg=latdeg,
              dzlay=dzlay, cld_frac=cld_frac, de_lgth=de_lgth, alpha=alpha)
    for n, v in flags.items():
        setattr(a, n, int(v))
    return _call(a, alpha, stream, sync)
