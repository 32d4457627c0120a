"""Seed part of ``GFS_rad_time_vary_timestep_init`` on the GPU.

Mirrors physics/Interstitials/UFS_SCM_NEPTUNE/GFS_rad_time_vary.fv3.F90:59-84:
when (lsswr or lslwr) and (isubc_lw == 2 or isubc_sw == 2), the McICA seeds
of every column are either copied from ``rseeds`` (lrseeds) or drawn for the
whole cubed-sphere face from one Mersenne-twister stream seeded with
``mod(nint(100 sqrt(sec)), ipsdlim) + 1 + ipsd0`` and picked by the column's
grid indices.  ``icsdlw`` is what ``rrtmg_lw_run`` takes as ``icseed``.

Arrays are int32 numpy arrays (host memory) or torch CUDA tensors (device
memory); the outputs are filled in place.  Returns ``(errmsg, errflg)`` like
the Fortran.  Runs in ``librrtmg_lw_gpu.so`` (``rrtmg_lw_gpu_seeds``).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from .rrtmg_lw import _is_device, lib, torch_stream


def gfs_rad_time_vary_seeds(lrseeds, rseeds, lslwr, lsswr, isubc_lw, isubc_sw, icsdsw, icsdlw, cnx, cny,
                            isc, jsc, imap, jmap, sec, ipsd0, ipsdlim, *, stream=None, sync=True):
    """``rseeds`` is the (n, 2) Fortran array, i.e. a C-contiguous (2, n) array."""
    n = int(icsdsw.shape[0])
    a = abi.SeedArgs(sec=float(sec), lslwr=int(bool(lslwr)), lsswr=int(bool(lsswr)), isubc_lw=int(isubc_lw),
                     isubc_sw=int(isubc_sw), lrseeds=int(bool(lrseeds)), ipsd0=int(ipsd0), ipsdlim=int(ipsdlim),
                     cnx=int(cnx), cny=int(cny), isc=int(isc), jsc=int(jsc), n=n,
                     ld_rseeds=int(rseeds.shape[-1]) if rseeds is not None else 0)
    for name, v in (("imap", imap), ("jmap", jmap), ("rseeds", rseeds), ("icsdsw", icsdsw), ("icsdlw", icsdlw)):
        setattr(a, name, abi._ptr(v, C.c_int32))
    device = _is_device(icsdsw)
    st = torch_stream(stream, icsdsw)
    x = abi.ExecArgs(memory=abi.DEVICE if device else abi.HOST,
                     stream=None if st is None else C.c_void_p(st), sync=int(sync))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_seeds(C.byref(a), C.byref(x), msg, 512)
    return msg.value.decode(), rc
