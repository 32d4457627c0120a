"""``rrtmg_lw_post_run`` on the GPU (physics/Radiation/RRTMG/rrtmg_lw_post.F90:13-77).

Maps the run's heating rates onto the model's levels (``htrlw(:,k) =
htlwc(:,k+kd)`` for k <= lm, the lm-th value repeated above), the clear-sky
ones into ``lwhc`` when ``lwhtr``, and copies ``tsfa`` into ``tsflw`` and
``sfcflw%dnfxc`` into ``sfcdlw``.  Called on the device-resident outputs of
``rrtmg_lw_run`` it keeps the heating-rate arrays on the device.

Arrays are Fortran-ordered ``(im[, levels])`` fields, ``sfcflw`` the (im, 4)
record array of the run; numpy (host) or torch CUDA tensors (device).
Returns ``(errmsg, errflg)``.  Runs in ``librrtmg_lw_gpu.so``
(``rrtmg_lw_gpu_post``).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from .rrtmg_lw import _is_device, lib, torch_stream


def rrtmg_lw_post_run(im, levs, ltp, lm, kd, lslwr, lwhtr, tsfa, htlwc, htlw0, sfcflw, tsflw, sfcdlw, htrlw,
                      lwhc, *, stream=None, sync=True):
    a = abi.PostArgs(im=int(im), levs=int(levs), ltp=int(ltp), lm=int(lm), kd=int(kd), lslwr=int(bool(lslwr)),
                     lwhtr=int(bool(lwhtr)))
    for n, v in (("tsfa", tsfa), ("htlwc", htlwc), ("htlw0", htlw0), ("sfcflw", sfcflw), ("tsflw", tsflw),
                 ("sfcdlw", sfcdlw), ("htrlw", htrlw), ("lwhc", lwhc)):
        abi._check_dtype(n, v, "f8")
        setattr(a, n, abi._ptr(v, C.c_double))
    st = torch_stream(stream, htrlw)
    x = abi.ExecArgs(memory=abi.DEVICE if _is_device(htrlw) else abi.HOST,
                     stream=None if st is None else C.c_void_p(st), sync=int(sync))
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_lw_gpu_post(C.byref(a), C.byref(x), msg, 512)
    return msg.value.decode(), rc
