"""Host-side checks of the learned gas optics' checkpoint wrappers (no GPU):
a training state of the wrong size is refused before the library is called,
and the checkpoint file keeps every field the C entry points exchange."""
import numpy as np
import pytest

from ccpp_physics_b200 import surrogate as sg


def test_set_state_refuses_wrong_sizes():
    ok = np.zeros(sg.NSTATE, dtype=np.float32)
    with pytest.raises(ValueError, match="training state"):
        sg.set_state(ok[:-1], ok, ok, 0, np.zeros(sg.NORM, dtype=np.float32))
    with pytest.raises(ValueError, match="training state"):
        sg.set_state(ok, ok, ok, 0, np.zeros(sg.NORM - 1, dtype=np.float32))


def test_checkpoint_file_round_trip(tmp_path, monkeypatch):
    rng = np.random.default_rng(3)
    state = {k: rng.standard_normal(sg.NSTATE).astype(np.float32) for k in ("params", "m", "v")}
    state.update(step=1234, norm=rng.standard_normal(sg.NORM).astype(np.float32))
    got = {}
    monkeypatch.setattr(sg, "get_state", lambda: state)
    monkeypatch.setattr(sg, "set_state", lambda p, m, v, step, norm: got.update(p=p, m=m, v=v, step=step, norm=norm))
    path = tmp_path / "ckpt.npz"
    sg.save_checkpoint(path, note="test")
    d = sg.load_checkpoint(path)
    assert str(d["note"]) == "test"
    for a, b in (("p", "params"), ("m", "m"), ("v", "v"), ("norm", "norm")):
        assert np.array_equal(got[a], state[b]), b
    assert got["step"] == 1234
