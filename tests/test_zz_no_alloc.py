"""GPU test of rrtmg_lw_gpu_run_noalloc, the entry point that allocates no
device memory.

It exists for callers that cannot let a library allocate during a run:
host models that give (nearly) all GPU memory to their own pool allocator
at start-up, and time-step loops that must not call cudaMalloc/cudaFree
because those calls synchronize the device.  The entry point takes its
scratch from a fixed array inside the library (made resident by
rrtmg_lw_gpu_init), so its results must equal those of the regular
device-memory entry point rrtmg_lw_gpu_run_ex.

The calls share that array and nothing clears it, so the test runs calls on
different inputs one after another: each later call finds the array as an
earlier call with other columns, seeds and clouds left it, and must still
match the regular entry point.  It also checks that the first call after
init takes no device memory, that a call too large for the array is refused
with the maximum, and that the refused overlaps are refused.  It runs alone
in a fresh process or after the other tests.
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


def _noalloc(lw, prof, out, precision=abi.FP64, flags=None):
    keep = []
    a = abi.make_run_args(prof, out, flags=flags, keep=keep)
    msg = C.create_string_buffer(512)
    rc = lw.lib().rrtmg_lw_gpu_run_noalloc(C.byref(a), precision, None, msg, 512)
    return rc, msg.value.decode()


def _profile(lw, npts, seed, clear_first=0, seed_base=None):
    """Device profile of npts columns; the first clear_first columns made
    cloud-free, McICA seeds seed_base + 7 i when given (else the column
    index)."""
    prof = synthetic.make_profiles(npts, 127, seed=seed)
    if clear_first:
        for k in ("cld_cf", "cld_lwp", "cld_iwp"):
            prof[k][:, :clear_first] = 0.0
    if seed_base is not None:
        prof["icseed"] = (seed_base + 7 * np.arange(npts)).astype(np.int32)
    return lw.to_device(prof)


def _check(out, ref, what):
    for k in ("topflx", "sfcflx", "flxprf"):
        a, b = out[k].cpu().numpy(), ref[k].cpu().numpy()
        rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
        assert rel <= FLUX_RTOL, (what, k, rel)
    for k in ("hlwc", "hlw0", "cldtau"):
        a, b = out[k].cpu().numpy(), ref[k].cpu().numpy()
        rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1.0))
        assert rel <= FLUX_RTOL, (what, k, rel)


@pytest.mark.parametrize("precision", [abi.FP64, abi.FP32])
def test_noalloc_matches_regular_entry_point(lib, precision):
    import torch
    prec = {abi.FP64: "fp64", abi.FP32: "fp32"}[precision]
    # three different calls in a row: a large cloudy one, then a smaller one
    # whose first half is cloud-free (the first call's columns there were
    # cloudy) with other seeds, then the first inputs again
    cases = [("large cloudy", _profile(lib, 150, 4242)),
             ("half clear, other seeds", _profile(lib, 96, 777, clear_first=48, seed_base=1000003)),
             ("first inputs again", _profile(lib, 150, 4242))]
    refs = []
    for _, prof in cases:
        ref = abi.alloc_outputs(prof["npts"], 127, hlw0=True, flxprf=True, like="cuda")
        msg, err = lib.run_profile(prof, ref, precision=prec)
        assert err == 0, msg
        refs.append(ref)
    torch.cuda.synchronize()
    for (what, prof), ref in zip(cases, refs):
        out = abi.alloc_outputs(prof["npts"], 127, hlw0=True, flxprf=True, like="cuda")
        out["cldtau"].fill_(123.0)   # every element must be written
        rc, msg = _noalloc(lib, prof, out, precision)
        assert rc == 0, msg
        _check(out, ref, what)


def test_noalloc_takes_no_device_memory(lib):
    import torch
    prof = _profile(lib, 64, 99)
    ref = abi.alloc_outputs(64, 127, hlw0=True, flxprf=True, like="cuda")
    msg, err = lib.run_profile(prof, ref)       # the kernels' modules are loaded by now
    assert err == 0, msg
    out = abi.alloc_outputs(64, 127, hlw0=True, flxprf=True, like="cuda")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, msg = _noalloc(lib, prof, out)
    assert rc == 0, msg
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # the 64 MiB array became resident at init: a call takes nothing more
    assert free0 - free1 < (16 << 20), (free0, free1)
    _check(out, ref, "after init")


def test_noalloc_rejects_too_many_columns(lib):
    npts, nlay = 512, 127
    prof = lib.to_device(synthetic.make_profiles(npts, nlay, seed=7))
    out = abi.alloc_outputs(npts, nlay, hlw0=True, like="cuda")
    rc, msg = _noalloc(lib, prof, out)
    assert rc == 1
    assert "at most" in msg and "columns" in msg, msg


@pytest.mark.parametrize("flags,word", [(dict(iovr=3), "iovr=3"), (dict(isubclw=0), "isubclw=0")])
def test_noalloc_refuses_other_cloud_treatments(lib, flags, word):
    prof = _profile(lib, 8, 5)
    out = abi.alloc_outputs(8, 127, hlw0=True, like="cuda")
    rc, msg = _noalloc(lib, prof, out, flags=flags)
    assert rc == 1 and word in msg, msg
