"""GPU test of rrtmg_lw_gpu_run_noalloc, the entry point that allocates no
device memory.

It exists for callers that cannot let a library allocate during a run:
host models that give (nearly) all GPU memory to their own pool allocator
at start-up, and time-step loops that must not call cudaMalloc/cudaFree
because those calls synchronize the device.  The entry point takes its
scratch from a fixed array inside the library, so its results must equal
those of the regular device-memory entry point; this test checks that, on
two calls in a row (the second call reuses the array as the first left it),
and that a call too large for the fixed array is refused with a clear
error.  It runs alone in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from ccpp_physics_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

FLUX_RTOL = 1e-10   # the tolerance of the FP64 parity tests


@pytest.fixture(scope="module")
def lib():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ccpp_physics_b200 import rrtmg_lw as lw
    rc, msg = lw.rlwinit(device=0)
    assert rc == 0, msg
    L = lw.lib()
    L.rrtmg_lw_gpu_run_noalloc.argtypes = [C.POINTER(abi.RunArgs), C.c_int32, C.c_void_p, C.c_char_p, C.c_int32]
    L.rrtmg_lw_gpu_run_noalloc.restype = C.c_int
    return lw


def _noalloc(lw, prof, out, precision=abi.FP64):
    keep = []
    a = abi.make_run_args(prof, out, keep=keep)
    msg = C.create_string_buffer(512)
    rc = lw.lib().rrtmg_lw_gpu_run_noalloc(C.byref(a), precision, None, msg, 512)
    return rc, msg.value.decode()


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32])
def test_noalloc_matches_regular_entry_point(lib, precision):
    import torch
    prec = {abi.FP64: "fp64", abi.FP32: "fp32"}[precision]
    npts, nlay = 96, 127
    prof = lib.to_device(synthetic.make_profiles(npts, nlay, seed=4242))
    ref = abi.alloc_outputs(npts, nlay, hlw0=True, flxprf=True, like="cuda")
    msg, err = lib.run_profile(prof, ref, precision=prec)
    assert err == 0, msg
    torch.cuda.synchronize()
    for call in range(2):
        out = abi.alloc_outputs(npts, nlay, hlw0=True, flxprf=True, like="cuda")
        rc, msg = _noalloc(lib, prof, out, precision)
        assert rc == 0, msg
        for k in ("topflx", "sfcflx", "flxprf"):
            a, b = out[k].cpu().numpy(), ref[k].cpu().numpy()
            rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
            assert rel <= FLUX_RTOL, (call, k, rel)
        for k in ("hlwc", "hlw0", "cldtau"):
            a, b = out[k].cpu().numpy(), ref[k].cpu().numpy()
            rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))
            assert rel <= FLUX_RTOL, (call, k, rel)


def test_noalloc_rejects_too_many_columns(lib):
    npts, nlay = 512, 127
    prof = lib.to_device(synthetic.make_profiles(npts, nlay, seed=7))
    out = abi.alloc_outputs(npts, nlay, hlw0=True, like="cuda")
    rc, msg = _noalloc(lib, prof, out)
    assert rc == 1
    assert "at most" in msg and "columns" in msg, msg
