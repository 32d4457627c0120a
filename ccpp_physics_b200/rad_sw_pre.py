"""``rad_sw_pre_run`` on the GPU (physics/Radiation/RRTMG/rad_sw_pre.F90:14-51).

Gathers the daytime points of a call: ``idxday(1:nday)`` lists, in
increasing order, the 1-based columns with ``coszen >= 0.0001`` and the rest
of ``idxday`` is zero; with ``lsswr`` false, ``nday = 0`` and ``idxday = 0``.
``coszen`` and ``idxday`` are (im) arrays: numpy (host) or torch CUDA tensors
(device; the ``idxday`` written then feeds ``rrtmg_sw_run`` on the device as
``idxday[:nday]``).  ``nday`` comes back to the host, so the call waits for
its stream.  Returns ``(nday, errmsg, errflg)``.  Runs in
``librrtmg_lw_gpu.so`` (``rrtmg_sw_gpu_pre``).
"""
from __future__ import annotations

import ctypes as C

from . import abi
from .rrtmg_lw import _is_device, torch_stream
from .rrtmg_sw import SwExec, SwPreArgs, lib


def rad_sw_pre_run(im, lsswr, coszen, idxday, *, stream=None):
    abi._check_dtype("coszen", coszen, "f8")
    abi._check_dtype("idxday", idxday, "i4")
    nday = C.c_int32(0)
    a = SwPreArgs(im=int(im), lsswr=int(bool(lsswr)), coszen=abi._ptr(coszen, C.c_double),
                  nday=C.pointer(nday), idxday=abi._ptr(idxday, C.c_int32))
    st = torch_stream(stream, idxday)
    x = SwExec(precision=0, memory=abi.DEVICE if _is_device(idxday) else abi.HOST,
               stream=None if st is None else C.c_void_p(st), sync=1)
    msg = C.create_string_buffer(512)
    rc = lib().rrtmg_sw_gpu_pre(C.byref(a), C.byref(x), msg, 512)
    return nday.value, msg.value.decode(), rc
