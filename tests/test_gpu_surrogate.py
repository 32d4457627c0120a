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
