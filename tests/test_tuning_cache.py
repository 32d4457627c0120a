"""The autotuner's JSON cache and rrtmg_lw_gpu_set_tuning, on the CPU.

rrtmg_lw_gpu_set_tuning only records the default launch shape (no device
work), so its checks run without a GPU.  The cache logic of
rrtmg_lw.autotune is exercised with the timing call replaced by a fake: a
miss times once and writes the choice under its (GPU, layer count,
precision) key, a hit sets that shape without timing."""
import ctypes as C
import json

import numpy as np
import pytest

from ccpp_physics_b200 import abi
from ccpp_physics_b200 import rrtmg_lw as lw


def test_set_tuning_checks_and_clears():
    lw.set_tuning(127, "fp32", {"rt_warps": 2, "gas_per_sm": 3, "chunk_cols": 4096})
    lw.set_tuning(127, "fp32", None)            # back to the built-in default
    lw.set_tuning(64, "fp64", {"rt_warps": 0})  # 0 = keep the default of that field
    lw.set_tuning(64, "fp64", None)
    with pytest.raises(lw.RRTMGLWError, match="rt_warps must be 1, 2 or 4"):
        lw.set_tuning(127, "fp32", {"rt_warps": 3})
    with pytest.raises(lw.RRTMGLWError, match="negative"):
        lw.set_tuning(127, "fp32", {"chunk_cols": -1})
    with pytest.raises(lw.RRTMGLWError, match="nlay must be 1..255"):
        lw.set_tuning(0, "fp32", None)


def test_autotune_cache_miss_then_hit(tmp_path, monkeypatch):
    L = lw.lib()
    timed = []

    def fake_autotune(arr, n, precision, stream, sample, best, ms, msg, mlen):
        timed.append(precision)
        b = best._obj                                   # the byref() arguments of the real call
        b.rt_warps, b.gas_per_sm, b.chunk_cols, b.use_graph = 2, 3, 8192, 0
        ms._obj.value = 12.5
        return 0

    monkeypatch.setattr(L, "rrtmg_lw_gpu_autotune", fake_autotune, raising=False)
    monkeypatch.setattr(lw, "block_args", lambda prof, out, sizes: ([], []))
    set_calls = []
    monkeypatch.setattr(lw, "set_tuning", lambda nlay, prec, t: set_calls.append((nlay, prec, dict(t))))
    prof = {"nlay": 127, "plyr": np.zeros((127, 8))}
    cache = tmp_path / "tuning.json"

    t, ms = lw.autotune(prof, {}, [8], precision="surrogate", cache=str(cache), device_name="NVIDIA B200")
    assert timed == [abi.SURROGATE] and set_calls == []
    assert t == {"rt_warps": 2, "gas_per_sm": 3, "chunk_cols": 8192, "use_graph": 0} and ms == 12.5
    table = json.loads(cache.read_text())
    assert list(table) == ["NVIDIA B200|nlay=127|surrogate"]

    t2, ms2 = lw.autotune(prof, {}, [8], precision="surrogate", cache=str(cache), device_name="NVIDIA B200")
    assert timed == [abi.SURROGATE]                     # the hit did not time again
    assert (t2, ms2) == (t, ms)
    assert set_calls == [(127, "surrogate", t)]         # and made the shape the default

    lw.autotune(prof, {}, [8], precision="fp64", cache=str(cache), device_name="NVIDIA B200")
    lw.autotune(prof, {}, [8], precision="surrogate", cache=str(cache), device_name="Other GPU")
    assert len(timed) == 3 and len(json.loads(cache.read_text())) == 3


def test_autotune_cache_rejects_a_non_object(tmp_path):
    cache = tmp_path / "bad.json"
    cache.write_text("[1, 2]")
    with pytest.raises(lw.RRTMGLWError, match="not a tuning cache"):
        lw.autotune({"nlay": 127, "plyr": np.zeros((1, 1))}, {}, [1], cache=str(cache), device_name="x")
