"""CPU tests of the RRTMG-SW pieces that need no GPU: the coefficient tables
extracted from radsw_datatb.f, the CPU restatement of rrtmg_sw_run
(physics/Radiation/RRTMG/radsw_main.F90) checked against identities the
reference's arithmetic implies, its sub-column generator against numpy's
independent MT19937, and the C ABI (exports, struct layout, error paths)."""
import ctypes as C
import hashlib
import json
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from ccpp_physics_b200 import rrtmg_sw as sw, synthetic

ROOT = os.path.join(os.path.dirname(__file__), "..")
DATA = os.path.join(ROOT, "ccpp_physics_b200", "data")


def _tables():
    blob = np.fromfile(os.path.join(DATA, "rrtmg_sw_tables.bin"), "<f8")
    man = json.load(open(os.path.join(DATA, "rrtmg_sw_tables.json")))
    return blob, man


def test_table_blob_checksum_and_literals():
    blob, man = _tables()
    raw = open(os.path.join(DATA, "rrtmg_sw_tables.bin"), "rb").read()
    assert hashlib.sha256(raw).hexdigest() == man["sha256"]
    hdr = open(os.path.join(DATA, "rrtmg_sw_table_layout.h")).read()
    assert man["sha256"] in hdr and str(man["ndouble"]) in hdr and blob.size == man["ndouble"]
    A = man["arrays"]
    g = lambda n, i=0: blob[A[n]["offset"] + i]
    # literals as written in radsw_datatb.f
    assert g("strrat", 6) == 3.63328e-2          # strrat(22), o2adj-scaled
    assert g("specwt", 1) == 4.0 and g("layreffr", 13) == 49 and g("ibx", 13) == 7
    assert g("scalekur") == 50.15 / 48.37
    assert g("b23_givfac") == 1.029 and g("a0r") == 3.07e-3 and g("a1s") == 1.5
    assert g("sfluxref01") == 3.65113 and g("preflog") == 6.96
    assert g("b24_rayla") == 0.1368516e-06 and g("b16_rayl") == 2.91e-10
    assert A["b17_absb"]["shape"] == [1175, 12] and A["b20_absa"]["shape"] == [65, 10]
    assert np.isfinite(blob).all()


@pytest.fixture(scope="module")
def osw():
    from oracle import oracle_sw
    rc, msg = oracle_sw.rswinit()
    assert rc == 0, msg
    return oracle_sw


def _profile(npts=24, nlay=40, seed=5, **kw):
    prof = synthetic.make_profiles(npts, nlay, seed=seed, cloudy=kw.pop("cloudy", True))
    return sw.add_sw_inputs(prof, seed=seed, **kw)


def test_oracle_identities(osw):
    prof = _profile(32, 60, night_fraction=0.25, precip=True)
    out = sw.alloc_outputs(32, 60, hswb=True, flxprf=True)
    rc, msg = osw.run(prof, out)
    assert rc == 0, msg
    day = prof["idxday"] - 1
    night = np.setdiff1d(np.arange(32), day)
    assert night.size and day.size
    for k in ("hswc", "hsw0", "cldtau"):
        assert not out[k][:, night].any(), k
    assert not out["topflx"][night].any() and not out["sfcflx"][night].any()
    # TOA downward flux is the solar source: s0fac * cosz * sum(sfluxzen)
    for ipt, j in enumerate(day[:6], start=1):
        _, _, sf, _ = osw.gas_optics(prof, ipt)
        want = (prof["solcon"] / 1368.22) * prof["cosz"][j] * sf.sum()
        assert abs(out["topflx"][j, 1] - want) <= 1e-12 * want
    # band heating rates add up to the total-sky rate; profiles end in the records
    assert np.allclose(out["hswb"].sum(0), out["hswc"], rtol=0, atol=1e-9 * np.abs(out["hswc"]).max())
    fp = out["flxprf"]
    assert np.array_equal(fp[0, day], out["sfcflx"][day][:, [0, 1, 2, 3]])
    assert np.array_equal(fp[-1, day, 0], out["topflx"][day, 0])
    # energy: absorbed = down at TOA - up at TOA - (down - up) at the surface >= 0
    absorbed = out["topflx"][day, 1] - out["topflx"][day, 0] - (out["sfcflx"][day, 1] - out["sfcflx"][day, 0])
    assert (absorbed > 0).all()


def test_oracle_clear_sky_total_equals_clear(osw):
    prof = _profile(16, 30, cloudy=False)
    out = sw.alloc_outputs(16, 30, flxprf=True)
    assert osw.run(prof, out)[0] == 0
    assert np.array_equal(out["topflx"][:, 0], out["topflx"][:, 2])
    assert np.array_equal(out["sfcflx"][:, :2], out["sfcflx"][:, 2:])
    assert np.array_equal(out["hswc"], out["hsw0"]) and not out["cldtau"].any()


def _flip(prof):
    """The same columns with the layer order reversed (top_at_1 input)."""
    f = dict(prof)
    for k, v in prof.items():
        if isinstance(v, np.ndarray) and v.ndim == 2 and v.shape[0] == prof["nlay"]:
            f[k] = np.ascontiguousarray(v[::-1])
        elif isinstance(v, np.ndarray) and v.ndim == 3 and v.shape[1] == prof["nlay"]:
            f[k] = np.ascontiguousarray(v[:, ::-1])
    return f


def test_oracle_top_at_1_is_a_flip(osw):
    prof = _profile(12, 33, precip=True)
    a = sw.alloc_outputs(12, 33, hswb=True, flxprf=True)
    b = sw.alloc_outputs(12, 33, hswb=True, flxprf=True)
    assert osw.run(prof, a)[0] == 0
    assert osw.run(_flip(prof), b, flags=dict(top_at_1=1))[0] == 0
    for k in ("topflx", "sfcflx", "fdncmp"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("hswc", "hsw0", "cldtau"):
        assert np.array_equal(a[k], b[k][::-1]), k
    assert np.array_equal(a["hswb"], b["hswb"][:, ::-1]) and np.array_equal(a["flxprf"], b["flxprf"][::-1])


def _gfs_stream(seed, m):
    key = np.zeros(624, dtype=np.uint64)
    v = (4357 if seed == 0 else seed) & 0xFFFFFFFF
    for i in range(624):
        key[i] = v
        v = (v * 69069) & 0xFFFFFFFF
    bg = np.random.MT19937(0)
    bg.state = {"bit_generator": "MT19937", "state": {"key": key.astype(np.uint32), "pos": 624}}
    return bg.random_raw(m).astype(np.float64) / 4294967295.0


@pytest.mark.parametrize("iovr", [0, 1, 2, 3, 4, 5])
def test_oracle_mcica_against_numpy_twister(osw, iovr):
    """mcica_subcol (radsw_main.F90:1952-2212), g-major draws, on numpy's MT19937."""
    nlay, seed = 37, 1234567
    rng = np.random.default_rng(4)
    cldf = rng.uniform(0, 1, nlay) * (rng.uniform(0, 1, nlay) > 0.3)
    dz = rng.uniform(0.05, 1.5, nlay)
    alpha = rng.uniform(0, 1, nlay)
    bits = osw.mcica_bits(nlay, seed, iovr, cldf, dz=dz, de_lgth=2.0, alpha=alpha)
    if iovr == 2:
        cdf = np.repeat(_gfs_stream(seed, 112)[:, None], nlay, 1)
    elif iovr >= 3:
        st = _gfs_stream(seed, 2 * 112 * nlay)
        cdf = st[:112 * nlay].reshape(112, nlay).copy()
        cd2 = st[112 * nlay:].reshape(112, nlay)
        if iovr == 3:
            fac = np.zeros(nlay)
            fac[1:] = np.exp(-0.5 * (dz[1:] + dz[:-1]) / 2.0)
            for k in range(nlay - 2, -1, -1):
                cdf[:, k] = np.where(cd2[:, k] <= fac[k + 1], cdf[:, k + 1], cdf[:, k])
        else:
            for k in range(1, nlay):
                cdf[:, k] = np.where(cd2[:, k] < alpha[k], cdf[:, k - 1], cdf[:, k])
    else:
        cdf = _gfs_stream(seed, 112 * nlay).reshape(112, nlay)
        if iovr == 1:
            for k in range(1, nlay):
                tem1 = 1.0 - cldf[k - 1]
                cdf[:, k] = np.where(cdf[:, k - 1] > tem1, cdf[:, k - 1], cdf[:, k] * tem1)
    want = cdf >= (1.0 - cldf)[None, :]
    got = np.array([[(bits[n, k >> 5] >> (k & 31)) & 1 for k in range(nlay)] for n in range(112)], bool)
    assert np.array_equal(got, want)


def test_oracle_spcvrtc_overcast_and_clear_limits(osw):
    """spcvrtc (isubcsw=0) mixes clear and cloudy optics by cldfrc = cfrac/cf1:
    with every cloudy layer at cf = 1 it equals the McICA path (every
    sub-column cloudy there), and a clear column gives clear-sky fluxes."""
    prof = _profile(16, 30, precip=True)
    cf = prof["cld_cf"]
    prof["cld_cf"] = np.where(cf > 0, 1.0, 0.0)
    a = sw.alloc_outputs(16, 30, flxprf=True)
    b = sw.alloc_outputs(16, 30, flxprf=True)
    assert osw.run(prof, a, flags=dict(isubcsw=0))[0] == 0
    assert osw.run(prof, b, flags=dict(isubcsw=2))[0] == 0
    for k in ("topflx", "sfcflx", "fdncmp", "flxprf"):
        assert np.allclose(a[k], b[k], rtol=1e-13, atol=0), k
    clear = _profile(8, 30, cloudy=False)
    c = sw.alloc_outputs(8, 30)
    assert osw.run(clear, c, flags=dict(isubcsw=0))[0] == 0
    assert np.array_equal(c["topflx"][:, 0], c["topflx"][:, 2])


def test_sw_struct_layout_matches_header(tmp_path):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    structs = {"rrtmg_sw_run_args": sw.SwRunArgs, "rrtmg_sw_init_args": sw.SwInitArgs, "rrtmg_sw_exec": sw.SwExec,
               "rrtmg_sw_post_args": sw.SwPostArgs, "rrtmg_sw_pre_args": sw.SwPreArgs}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rrtmg_sw_gpu.h"', 'int main(void){']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                  check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_sw_run_before_init_reports_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU path")
    prof = _profile(2, 10)
    with pytest.raises(sw.RrtmgSwError, match="init"):
        sw.rrtmg_sw_run(prof, sw.alloc_outputs(2, 10))


def _golden_cases():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_sw_golden", os.path.join(ROOT, "tests", "golden",
                                                                                 "make_sw_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("name", ["sw_allsky_127lay", "sw_dcorr_127lay", "sw_gridmean_64lay"])
def test_oracle_reproduces_golden_fixture(osw, name):
    """Regression pin: the restatement still gives the committed outputs bit for bit."""
    g = _golden_cases()
    case = g.CASES[name]
    prof = g.profile(case)
    out = sw.alloc_outputs(case["npts"], case["nlay"], hswb=True, flxprf=True)
    assert osw.run(prof, out, flags=case["flags"])[0] == 0
    ref = np.load(os.path.join(ROOT, "tests", "golden", f"oracle_{name}.npz"))
    for k in ref.files:
        assert np.array_equal(out[k], ref[k]), k


def _post_case(rng, im, levs, ltp, lm, fill=7.0):
    """Inputs and filled outputs of rrtmg_sw_post_run, Fortran-ordered."""
    ins = dict(sfcalb1=rng.uniform(0, 1, im), sfcalb2=rng.uniform(0, 1, im), sfcalb3=rng.uniform(0, 1, im),
               sfcalb4=rng.uniform(0, 1, im), htswc=rng.normal(size=(lm + ltp, im)),
               htsw0=rng.normal(size=(lm + ltp, im)))
    outs = {n: np.full(im, fill) for n in ("nirbmdi", "nirdfdi", "visbmdi", "visdfdi", "nirbmui", "nirdfui",
                                           "visbmui", "visdfui", "sfcdsw", "sfcnsw")}
    outs.update(htrsw=np.full((levs, im), fill), swhc=np.full((levs, im), fill),
                scmpsw=rng.uniform(0, 500, (im, 6)), sfcfsw=rng.uniform(0, 900, (im, 4)),
                topfsw=rng.uniform(0, 1300, (im, 3)))
    return ins, outs


@pytest.mark.parametrize("nday", [3, 0])
def test_oracle_sw_post_restatement(osw, nday):
    """rrtmg_sw_post_run (rrtmg_sw_post.F90:52-127) against numpy statements."""
    rng = np.random.default_rng(11 + nday)
    im, levs, ltp, lm, kd = 13, 9, 1, 6, 1
    ins, outs = _post_case(rng, im, levs, ltp, lm)
    before = {k: v.copy() for k, v in outs.items()}
    osw.post(im, lm, levs, ltp, nday, lm, kd, True, True, *ins.values(), *outs.values())
    if nday:
        src = np.minimum(np.arange(levs), lm - 1) + kd
        assert np.array_equal(outs["htrsw"], ins["htswc"][src]) and np.array_equal(outs["swhc"], ins["htsw0"][src])
        c = before["scmpsw"]
        for j, (d, u, alb) in enumerate((("nirbmdi", "nirbmui", "sfcalb1"), ("nirdfdi", "nirdfui", "sfcalb2"),
                                         ("visbmdi", "visbmui", "sfcalb3"), ("visdfdi", "visdfui", "sfcalb4"))):
            assert np.array_equal(outs[d], c[:, 2 + j]) and np.array_equal(outs[u], c[:, 2 + j] * ins[alb])
        for k in ("scmpsw", "sfcfsw", "topfsw"):
            assert np.array_equal(outs[k], before[k]), k
    else:
        for k, v in outs.items():
            if k not in ("sfcdsw", "sfcnsw"):
                assert not v.any(), k
    f = outs["sfcfsw"]
    assert np.array_equal(outs["sfcnsw"], f[:, 1] - f[:, 0]) and np.array_equal(outs["sfcdsw"], f[:, 1])
    untouched = {k: v.copy() for k, v in outs.items()}
    osw.post(im, lm, levs, ltp, nday, lm, kd, False, True, *ins.values(), *outs.values())   # lsswr false
    assert all(np.array_equal(outs[k], untouched[k]) for k in outs)


def test_sw_post_entry_point_validation():
    """Host-side checks of rrtmg_sw_gpu_post (return before any CUDA call)."""
    L = sw.lib()
    x = sw.SwExec(memory=0, sync=1)
    m = C.create_string_buffer(256)
    assert L.rrtmg_sw_gpu_post(None, C.byref(x), m, 256) == 1 and b"null" in m.value
    p = sw.SwPostArgs(im=2, levs=3, ltp=0, nday=1, lm=2, kd=1, lsswr=1)
    assert L.rrtmg_sw_gpu_post(C.byref(p), C.byref(x), m, 256) == 1 and b"kd <= ltp" in m.value
    p.lsswr = 0                                   # rrtmg_sw_post.F90:52: nothing to do
    assert L.rrtmg_sw_gpu_post(C.byref(p), C.byref(x), m, 256) == 0
    buf = (C.c_double * 64)()
    dp = C.cast(buf, C.POINTER(C.c_double))
    p = sw.SwPostArgs(im=2, levs=3, ltp=0, nday=0, lm=9, kd=5, lsswr=1)   # lm, kd unread at night
    for n in sw.POST_OUTPUT_FIELDS:
        if n != "topfsw":
            setattr(p, n, dp)
    assert L.rrtmg_sw_gpu_post(C.byref(p), C.byref(x), m, 256) == 1 and b"topfsw" in m.value
    p.nday, p.lm, p.kd = 2, 3, 0
    assert L.rrtmg_sw_gpu_post(C.byref(p), C.byref(x), m, 256) == 1 and b"sfcalb" in m.value
    p.im = 0
    p.sfcalb1 = p.sfcalb2 = p.sfcalb3 = p.sfcalb4 = p.htswc = p.htsw0 = dp
    assert L.rrtmg_sw_gpu_post(C.byref(p), C.byref(x), m, 256) == 0   # no columns: nothing to do


def test_oracle_sw_pre_restatement(osw):
    """rad_sw_pre_run (rad_sw_pre.F90:36-49) against numpy, with values on the
    0.0001 threshold and either side of it."""
    rng = np.random.default_rng(5)
    im = 3000
    cz = rng.uniform(-1, 1, im)
    cz[::7] = 1e-4
    cz[1::11] = np.nextafter(1e-4, 0)
    cz[2::13] = np.nextafter(1e-4, 1)
    nday, idx = osw.pre(im, True, cz)
    want = np.nonzero(cz >= 1e-4)[0] + 1
    assert nday == len(want) and np.array_equal(idx[:nday], want) and not idx[nday:].any()
    nday, idx = osw.pre(im, False, cz)
    assert nday == 0 and not idx.any()


def test_sw_pre_entry_point_validation():
    L = sw.lib()
    x = sw.SwExec(memory=0, sync=1)
    m = C.create_string_buffer(256)
    nd = C.c_int32(5)
    assert L.rrtmg_sw_gpu_pre(None, C.byref(x), m, 256) == 1 and b"null" in m.value
    p = sw.SwPreArgs(im=-1, lsswr=1, nday=C.pointer(nd))
    assert L.rrtmg_sw_gpu_pre(C.byref(p), C.byref(x), m, 256) == 1 and b"im >= 0" in m.value
    p.im = 4
    assert L.rrtmg_sw_gpu_pre(C.byref(p), C.byref(x), m, 256) == 1 and b"required" in m.value
    p.im = 0                                      # no columns: nday = 0, nothing else to do
    assert L.rrtmg_sw_gpu_pre(C.byref(p), C.byref(x), m, 256) == 0 and nd.value == 0


def test_pre_post_wrappers_refuse_wrong_dtypes():
    """A wrong element type would be read through the wrong pointer type: the
    Python mirrors refuse it before any call."""
    from ccpp_physics_b200.rad_sw_pre import rad_sw_pre_run
    from ccpp_physics_b200.rrtmg_sw_post import rrtmg_sw_post_run
    with pytest.raises(TypeError, match="idxday must be int32"):
        rad_sw_pre_run(4, True, np.ones(4), np.zeros(4, np.int64))
    with pytest.raises(TypeError, match="coszen must be float64"):
        rad_sw_pre_run(4, True, np.ones(4, np.float32), np.zeros(4, np.int32))
    z = np.zeros(2)
    with pytest.raises(TypeError, match="sfcalb1 must be float64"):
        rrtmg_sw_post_run(2, 1, 1, 0, 1, 1, 0, True, False, z.astype(np.float32), *[z] * 20)
