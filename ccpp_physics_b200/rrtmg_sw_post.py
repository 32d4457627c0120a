"""``rrtmg_sw_post_run`` on the GPU (physics/Radiation/RRTMG/rrtmg_sw_post.F90:13-129).

With daytime points (``nday > 0``) it maps the run's heating rates onto the
model's levels (``htrsw(:,k) = htswc(:,k+kd)`` for k <= lm, the lm-th value
repeated above), the clear-sky ones into ``swhc`` when ``swhtr``, and splits
the surface components of ``scmpsw`` into the four downward fields and their
products with ``sfcalb1..4``; with none it zeroes those outputs and the
``sfcfsw``, ``topfsw`` and ``scmpsw`` records.  Then ``sfcnsw`` and ``sfcdsw``
are the net and downward surface fluxes of ``sfcfsw``.  Called on the
device-resident outputs of ``rrtmg_sw_run`` it keeps them on the device.

Arrays are Fortran-ordered ``(im[, levels])`` fields; the records are the
run's (im, 6) ``cmpfsw``, (im, 4) ``sfcfsw`` and (im, 3) ``topfsw`` arrays;
numpy (host) or torch CUDA tensors (device).  Returns ``(errmsg, errflg)``.
Runs in ``librrtmg_lw_gpu.so`` (``rrtmg_sw_gpu_post``).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from .rrtmg_lw import _is_device, torch_stream
from .rrtmg_sw import POST_INPUT_FIELDS, POST_OUTPUT_FIELDS, SwExec, SwPostArgs, lib


def rrtmg_sw_post_run(im, levr, levs, ltp, nday, lm, kd, lsswr, swhtr, sfcalb1, sfcalb2, sfcalb3, sfcalb4,
                      htswc, htsw0, nirbmdi, nirdfdi, visbmdi, visdfdi, nirbmui, nirdfui, visbmui, visdfui,
                      sfcdsw, sfcnsw, htrsw, swhc, scmpsw, sfcfsw, topfsw, *, stream=None, sync=True):
    vals = locals()
    a = SwPostArgs(im=int(im), levr=int(levr), levs=int(levs), ltp=int(ltp), nday=int(nday), lm=int(lm),
                   kd=int(kd), lsswr=int(bool(lsswr)), swhtr=int(bool(swhtr)))
    for n in POST_INPUT_FIELDS + POST_OUTPUT_FIELDS:
        abi._check_dtype(n, vals[n], "f8")
        setattr(a, n, abi._ptr(vals[n], C.c_double))
    st = torch_stream(stream, sfcfsw)
    x = SwExec(precision=0, memory=abi.DEVICE if _is_device(sfcfsw) else abi.HOST,
               stream=None if st is None else C.c_void_p(st), sync=int(sync))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_sw_gpu_post(C.byref(a), C.byref(x), msg, 512)
    return msg.value.decode(), rc
