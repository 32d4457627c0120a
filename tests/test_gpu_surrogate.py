"""GPU tests of the learned gas optics (tcgen05 BF16 kernels in
csrc/lw_mlp.cu): forward pass and gradients against the CPU oracle
(oracle/mlp_oracle.py), training, the surrogate column path against the FP64
path, the out-of-envelope fallback to taumol, and what the trained network
gains over the path without it."""
import numpy as np
import pytest

from ccpp_physics_b200 import abi, synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sg():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ccpp_physics_b200 import rrtmg_lw as lw
    from ccpp_physics_b200 import surrogate
    rc, msg = lw.rlwinit(device=0)
    assert rc == 0, msg
    return surrogate


@pytest.fixture(scope="module")
def small_set(sg):
    """~64k layer samples from plain taumol, with their normalisation."""
    feats, targ = sg.make_dataset(512 * 127, seed=202)
    norm = sg.normalisation(feats, targ)
    return feats, targ, norm


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_forward_matches_oracle(sg, small_set):
    from oracle import mlp_oracle as mo
    feats, targ, norm = small_set
    sg.init(norm, seed=3)
    w, n = sg.get_weights()
    x = feats[:1000]
    y = sg.forward(x).cpu().numpy()
    ref = mo.forward(mo.normalise(x.cpu().numpy(), n), mo.unpack(w))["y"]
    keep = np.setdiff1d(np.arange(288), mo.PAD)
    assert np.all(y[:, mo.PAD] == y[:, mo.PAD])          # written (not NaN)
    assert _rel(y[:, keep], ref[:, keep]) < 5e-3
    assert np.max(np.abs(y[:, keep] - ref[:, keep])) < 5e-2 * max(1.0, np.max(np.abs(ref)))


def test_gradients_match_oracle(sg, small_set):
    from oracle import mlp_oracle as mo
    feats, targ, norm = small_set
    sg.init(norm, seed=5)
    y = sg.normalise_targets(targ, norm)
    B = 512
    g, loss = sg.grads(feats, y, B)
    w, n = sg.get_weights()
    ref_loss, ref = mo.loss_and_grads(mo.normalise(feats[:B].cpu().numpy(), n), y[:B].cpu().numpy().astype(np.float64),
                                      mo.unpack(w))
    rg = mo.pack_grads(ref)
    assert abs(loss - ref_loss) <= 2e-3 * ref_loss
    parts = [(0, 1024), (1024, 17408), (17408, 17536), (17536, 54400), (54400, 54688)]
    for a, b in parts:
        assert _rel(g[a:b], rg[a:b]) < 3e-2, (a, b, _rel(g[a:b], rg[a:b]))


def test_training_reduces_loss(sg, small_set):
    feats, targ, norm = small_set
    sg.init(norm, seed=11)
    y = sg.normalise_targets(targ, norm)
    losses = sg.train(feats, y, epochs=6, batch=1024, lr=3e-3, lr_final=1e-4)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.25 * losses[0], losses


def test_training_checkpoint_resumes(sg, small_set, tmp_path):
    """A training checkpoint holds the FP32 parameters, both Adam moments, the
    step count and the normalisation: restored after other weights were
    loaded (which also resets the optimizer), it gives back the same state
    bit for bit and the same forward outputs, and training continues from
    its step."""
    feats, targ, norm = small_set
    sg.init(norm, seed=13)
    y = sg.normalise_targets(targ, norm)
    batch = 1024
    sg.train(feats, y, epochs=2, batch=batch, lr=3e-3, lr_final=1e-3)
    st = sg.get_state()
    steps = feats.shape[0] // batch
    assert st["step"] == 2 * steps
    assert np.any(st["m"] != 0) and np.any(st["v"] != 0)
    x = feats[:1024].contiguous()
    y0 = sg.forward(x).cpu().numpy()
    path = tmp_path / "ckpt.npz"
    sg.save_checkpoint(path)
    sg.init(norm, seed=99)                      # other weights and a fresh optimizer
    fresh = sg.get_state()
    assert fresh["step"] == 0 and not np.any(fresh["m"]) and not np.any(fresh["v"])
    sg.load_checkpoint(path)
    st2 = sg.get_state()
    for k in ("params", "m", "v", "norm"):
        assert np.array_equal(st[k], st2[k]), k
    assert st2["step"] == st["step"]
    assert np.array_equal(sg.forward(x).cpu().numpy(), y0)
    losses = sg.train(feats, y, epochs=1, batch=batch, lr=1e-3, lr_final=1e-4)
    assert np.all(np.isfinite(losses))
    assert sg.get_state()["step"] == 3 * steps


@pytest.fixture(scope="module")
def trained(sg):
    """The committed network, trained on the GPU by ccpp_physics_b200.train_surrogate."""
    d = sg.load()
    return d


def _run(lw, prof, precision, n, nlay):
    o = abi.alloc_outputs(n, nlay, hlw0=True, like="cuda")
    msg, err = lw.run_profile(prof, o, precision=precision)
    assert err == 0, msg
    return o


def _rmse(a, b):
    import torch
    return float(torch.sqrt(torch.mean((a - b) ** 2)).item())


def test_surrogate_path_meets_accuracy_bounds(sg, trained):
    """All-sky McICA columns the network never saw (generator seed 1): fluxes
    within 0.5 W/m2 RMSE and heating rates within 0.1 K/day RMSE of the FP64 path."""
    import torch
    from ccpp_physics_b200 import rrtmg_lw as lw
    n, nlay = 4096, 127
    prof = lw.to_device(synthetic.make_profiles(n, nlay, seed=1))
    sg.stats(reset=True)
    s = _run(lw, prof, "surrogate", n, nlay)
    fallback, mma_err = sg.stats()
    r = _run(lw, prof, "fp64", n, nlay)
    assert mma_err == 0
    assert fallback < 0.01 * n * nlay
    flux = _rmse(torch.cat([s["topflx"], s["sfcflx"]], 1), torch.cat([r["topflx"], r["sfcflx"]], 1))
    hr = _rmse(s["hlwc"], r["hlwc"])
    assert flux <= 0.5, flux
    assert hr <= 0.1, hr
    assert _rmse(s["hlw0"], r["hlw0"]) <= 0.1
    assert torch.equal(s["cldtau"], r["cldtau"]) or _rmse(s["cldtau"], r["cldtau"]) < 1e-5


@pytest.mark.parametrize("nlay", [64, 100])
def test_surrogate_path_short_columns(sg, trained, nlay):
    """Columns of fewer layers than the network's 128-row tile: the padding
    rows past a column's last 8-layer hand-off block must write nothing (the
    next column's hand-off follows), so two runs agree bit for bit and every
    column stays close to the FP64 path (a column whose hand-off was
    overwritten is off by tens of W/m2)."""
    import torch
    from ccpp_physics_b200 import rrtmg_lw as lw
    n = 2048
    prof = lw.to_device(synthetic.make_profiles(n, nlay, seed=5))
    s1 = _run(lw, prof, "surrogate", n, nlay)
    s2 = _run(lw, prof, "surrogate", n, nlay)
    r = _run(lw, prof, "fp64", n, nlay)
    for k in ("topflx", "sfcflx", "hlwc"):
        assert torch.equal(s1[k], s2[k]), k
    flux = torch.cat([s1["topflx"], s1["sfcflx"]], 1) - torch.cat([r["topflx"], r["sfcflx"]], 1)
    assert bool(torch.isfinite(flux).all())
    assert float(flux.abs().max()) <= 10.0, float(flux.abs().max())
    assert _rmse(flux, torch.zeros_like(flux)) <= 1.0
    assert _rmse(s1["hlwc"], r["hlwc"]) <= 0.2


def test_out_of_envelope_layers_fall_back_to_taumol(sg, trained):
    """Doubled CO2 (the training set holds 400 ppmv) puts every layer outside
    the envelope: every layer's optical depths and Planck fractions then come
    from plain FP32 taumol, the FP32 path's gas optics, so the result is the
    FP32 path's up to the learned-gas-optics path's FP16 copies (relative
    rounding 2^-11) of the optical depths, Planck fractions, transmittance
    records and up-sweep terms, and the order of its sums over g-points:
    fluxes within 3e-4 relative, heating rates within 0.01 K/day RMSE and
    5 % of max(|rate|, 1 K/day) everywhere, cloud optical depth equal.  The
    network's own error against FP32 taumol is ten times larger (flux RMSE
    ~0.1 W/m2, heating rates ~0.05 K/day)."""
    import torch
    from ccpp_physics_b200 import rrtmg_lw as lw
    n, nlay = 512, 127
    p = synthetic.make_profiles(n, nlay, seed=21)
    p["gasvmr_co2"] = p["gasvmr_co2"] * 2.0
    prof = lw.to_device(p)
    sg.stats(reset=True)
    s = _run(lw, prof, "surrogate", n, nlay)
    fallback, _ = sg.stats()
    assert fallback == n * nlay
    f = _run(lw, prof, "fp32", n, nlay)
    assert torch.equal(s["cldtau"], f["cldtau"])
    for k in ("topflx", "sfcflx"):
        rel = float(((s[k] - f[k]).abs() / f[k].abs()).max())
        assert rel <= 3e-4, (k, rel)
    for k in ("hlwc", "hlw0"):
        assert _rmse(s[k], f[k]) <= 1e-2, (k, _rmse(s[k], f[k]))
        d = float(((s[k] - f[k]).abs() / f[k].abs().clamp_min(1.0)).max())
        assert d <= 5e-2, (k, d)
    # only the upper half of every column outside: exactly those layers fall back
    p2 = synthetic.make_profiles(n, nlay, seed=21)
    p2["gasvmr_co2"][64:] *= 2.0
    sg.stats(reset=True)
    _run(lw, lw.to_device(p2), "surrogate", n, nlay)
    assert sg.stats()[0] == n * (nlay - 64)


def test_trained_network_gain(sg, trained):
    """What the trained network adds: against the same network untrained
    (random initial weights, same normalisation) its fluxes are far closer to
    FP64, and against plain taumol in FP32 (the path without it) it is faster."""
    import torch
    from ccpp_physics_b200 import rrtmg_lw as lw
    n, nlay = 16384, 127
    prof = lw.to_device(synthetic.make_profiles(n, nlay, seed=3))
    r = _run(lw, prof, "fp64", n, nlay)
    s = _run(lw, prof, "surrogate", n, nlay)
    err_trained = _rmse(torch.cat([s["topflx"], s["sfcflx"]], 1), torch.cat([r["topflx"], r["sfcflx"]], 1))

    def best_ms(precision):
        o = abi.alloc_outputs(n, nlay, hlw0=True, like="cuda")
        times = []
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            msg, err = lw.run_profile(prof, o, precision=precision)
            e1.record()
            torch.cuda.synchronize()
            assert err == 0, msg
            times.append(e0.elapsed_time(e1))
        return min(times)
    t_sg, t_fp32 = best_ms("surrogate"), best_ms("fp32")
    w, norm = sg.get_weights()
    sg.init(norm, seed=9)                       # untrained network
    u = _run(lw, prof, "surrogate", n, nlay)
    err_untrained = _rmse(torch.cat([u["topflx"], u["sfcflx"]], 1), torch.cat([r["topflx"], r["sfcflx"]], 1))
    sg.set_weights(w, norm)
    assert err_trained < 0.02 * err_untrained, (err_trained, err_untrained)
    assert t_sg < 0.9 * t_fp32, (t_sg, t_fp32)


def test_forward_wait_timeout_is_reported_and_recovers(sg, small_set):
    """Failure detection without a GPU fault: with the tensor-core wait limit
    at zero polls every wait of the forward kernel gives up at once.  The call
    must return the time-out error (and mma_error), the kernels must still
    wait for their MMAs and free their tensor memory, and with the default
    limit restored the next call runs and gives the same outputs as before."""
    import ctypes as C
    import torch
    feats, _, _ = small_set
    sg.load()                 # the committed network
    x = feats[:4096].contiguous()
    y_ref = sg.forward(x)
    L = sg._lib()
    L.rrtmg_lw_gpu_surrogate_wait_limit.argtypes = [C.c_int64]
    assert L.rrtmg_lw_gpu_surrogate_wait_limit(0) == 0
    try:
        y = torch.empty((x.shape[0], 288), dtype=torch.float32, device="cuda")
        msg = C.create_string_buffer(512)
        rc = L.rrtmg_lw_gpu_surrogate_forward(C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(y.data_ptr()),
                                              None, msg, 512)
        assert rc == 1 and "timed out" in msg.value.decode(), msg.value
        _, err = sg.stats(reset=True)
        assert err == 1
    finally:
        assert L.rrtmg_lw_gpu_surrogate_wait_limit(-1) == 0
    y2 = sg.forward(x)        # every SM allocates its tensor memory again
    assert torch.equal(y2, y_ref)
    _, err = sg.stats(reset=True)
    assert err == 0
