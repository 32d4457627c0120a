"""GPU tests of the batched physics-block entry point (rrtmg_lw_gpu_run_blocks),
its CUDA-graph replay and the launch-shape autotuner.

The reference host calls rrtmg_lw_run once per physics block
(radlw_main.F90:419); the batched call must give every column exactly the
result of that per-block call: bit-identical, since the same kernels do the
same arithmetic per column.
"""
import numpy as np
import pytest

from ccpp_physics_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

NLAY = 127
NCOLS = 700


@pytest.fixture(scope="module")
def lw():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ccpp_physics_b200 import rrtmg_lw
    rc, msg = rrtmg_lw.rlwinit(device=0)
    assert rc == 0, msg
    return rrtmg_lw


@pytest.fixture(scope="module")
def case(lw):
    sizes = synthetic.physics_blocks(NCOLS, seed=5)
    prof = lw.to_device(synthetic.make_profiles(NCOLS, NLAY, seed=77))
    return sizes, prof


def _outs():
    return abi.alloc_outputs(NCOLS, NLAY, hlw0=True, flxprf=True, like="cuda")


def _equal(a, b):
    import torch
    for k in a:
        assert torch.equal(a[k], b[k]), k


@pytest.mark.parametrize("precision", ["fp64", "fp32", "surrogate"])
def test_blocks_equal_one_call(lw, case, precision):
    """isubclw=2 seeds come from icseed, so the block split changes nothing
    (the learned gas optics included: its rows are independent)."""
    sizes, prof = case
    if precision == "surrogate":
        from ccpp_physics_b200 import surrogate
        surrogate.load()
    one, many = _outs(), _outs()
    msg, err = lw.run_profile(prof, one, precision=precision)
    assert err == 0, msg
    msg, err = lw.run_blocks(prof, many, sizes, precision=precision)
    assert err == 0, msg
    _equal(many, one)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_packed_blocks_equal_views(lw, case, precision):
    """Blocks held as separate (n_b, nlay) arrays (ldim = n_b, as a host that
    allocates each physics block separately passes them) give the results of
    the same blocks as views into one array, bit for bit."""
    sizes, prof = case
    views = _outs()
    assert lw.run_blocks(prof, views, sizes, precision=precision)[1] == 0
    pp = lw.pack_blocks(prof, sizes)
    po = lw.pack_blocks(_outs(), sizes)
    msg, err = lw.run_blocks(pp, po, sizes, precision=precision)
    assert err == 0, msg
    _equal(lw.unpack_blocks(po), views)


def test_blocks_equal_per_block_calls_isubclw1(lw, case):
    """isubclw=1 seeds are block-relative (140+i, radlw_main.F90:766-768):
    the batched call must equal one rrtmg_lw_run per block."""
    import torch
    sizes, prof = case
    many = _outs()
    flags = dict(prof["flags"], isubclw=1)
    p1 = dict(prof, flags=flags)
    msg, err = lw.run_blocks(p1, many, sizes)
    assert err == 0, msg
    c0 = 0
    for n in sizes[:12]:
        sub = {k: (v[..., c0:c0 + n].contiguous() if isinstance(v, torch.Tensor) else v) for k, v in p1.items()}
        sub["npts"] = int(n)
        o = abi.alloc_outputs(int(n), NLAY, hlw0=True, flxprf=True, like="cuda")
        msg, err = lw.run_profile(sub, o)
        assert err == 0, msg
        assert torch.equal(o["topflx"], many["topflx"][c0:c0 + n])
        assert torch.equal(o["hlwc"], many["hlwc"][:, c0:c0 + n])
        assert torch.equal(o["flxprf"], many["flxprf"][:, c0:c0 + n])
        c0 += int(n)


@pytest.mark.parametrize("shape", [dict(rt_warps=1), dict(rt_warps=2, chunk_cols=150),
                                   dict(rt_warps=4, gas_per_sm=1, chunk_cols=333)])
def test_launch_shapes_same_result(lw, case, shape):
    sizes, prof = case
    ref, o = _outs(), _outs()
    assert lw.run_blocks(prof, ref, sizes)[1] == 0
    msg, err = lw.run_blocks(prof, o, sizes, tuning=shape)
    assert err == 0, msg
    _equal(o, ref)


def test_graph_replay_tracks_inputs(lw, case):
    """A captured block set replays through the same pointers: results equal
    the eager call, also after the inputs change in place."""
    import torch
    sizes, prof = case
    prof = {k: (v.clone() if isinstance(v, torch.Tensor) else v) for k, v in prof.items()}
    g, ref = _outs(), _outs()
    for _ in range(2):                                   # capture, then replay
        msg, err = lw.run_blocks(prof, g, sizes, tuning=dict(use_graph=1))
        assert err == 0, msg
    assert lw.run_blocks(prof, ref, sizes)[1] == 0
    _equal(g, ref)
    prof["tlyr"] += 1.5
    prof["tlvl"] += 1.5
    msg, err = lw.run_blocks(prof, g, sizes, tuning=dict(use_graph=1))
    assert err == 0, msg
    assert lw.run_blocks(prof, ref, sizes)[1] == 0
    _equal(g, ref)


def test_autotune_picks_valid_shape(lw, case):
    sizes, prof = case
    o = _outs()
    best, ms = lw.autotune(prof, o, sizes, precision="fp32", sample_cols=400)
    assert best["rt_warps"] in (1, 2, 4) and best["chunk_cols"] >= 0 and ms > 0
    ref, o2 = _outs(), _outs()
    assert lw.run_blocks(prof, o2, sizes, precision="fp32")[1] == 0       # tuned default
    assert lw.run_blocks(prof, ref, sizes, precision="fp32", tuning=dict(rt_warps=4))[1] == 0
    _equal(o2, ref)


def test_run_blocks_errors(lw, case):
    import ctypes as C
    sizes, prof = case
    o = _outs()
    arr, keep = lw.block_args(prof, o, sizes)
    arr[3].nlay = 64
    arr[3].nlp1 = 65
    x = abi.ExecArgs(precision=abi.FP64, memory=abi.DEVICE, sync=1)
    msg = C.create_string_buffer(512)
    rc = lw.lib().rrtmg_lw_gpu_run_blocks(arr, len(arr), C.byref(x), None, msg, 512)
    assert rc == 1 and b"block 3" in msg.value
    x.memory = abi.HOST
    rc = lw.lib().rrtmg_lw_gpu_run_blocks(arr, len(arr), C.byref(x), None, msg, 512)
    assert rc == 1 and b"device memory" in msg.value
    msg2, err = lw.run_blocks(prof, o, sizes, tuning=dict(rt_warps=3))
    assert err == 1 and "rt_warps" in msg2
