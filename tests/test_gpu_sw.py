"""GPU parity tests of the RRTMG-SW path: the CUDA kernels through the C ABI
(rrtmg_sw_gpu_run_ex) against the CPU restatement of rrtmg_sw_run
(physics/Radiation/RRTMG/radsw_main.F90:493-1379) on identical inputs.

Bars (those of the longwave path): fluxes within 1e-10 relative; heating
rates within 1e-9 * max(|ref|, 1 K/day), since the GPU sums the g-point
fluxes in another order than the reference and heating rates difference
nearly equal fluxes; McICA flags are bit-exact, which the cloudy-column
fluxes expose (one flipped sub-column moves fluxes by far more than 1e-10).
"""
import numpy as np
import pytest

from ccpp_physics_b200 import rrtmg_sw as sw, synthetic

pytestmark = pytest.mark.gpu

FLUX_RTOL = 1e-10
HR_TOL = 1e-9


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sw.rswinit(device=0)
    return sw


@pytest.fixture(scope="module")
def osw():
    from oracle import oracle_sw
    rc, msg = oracle_sw.rswinit()
    assert rc == 0, msg
    return oracle_sw


def _profile(npts, nlay, seed, **kw):
    prof = synthetic.make_profiles(npts, nlay, seed=seed, cloudy=kw.pop("cloudy", True))
    return sw.add_sw_inputs(prof, seed=seed, **kw)


def _flip(prof):
    """The same columns with the layer order reversed (top_at_1 input)."""
    f = dict(prof)
    for k, v in prof.items():
        if isinstance(v, np.ndarray) and v.ndim == 2 and v.shape[0] == prof["nlay"]:
            f[k] = np.ascontiguousarray(v[::-1])
        elif isinstance(v, np.ndarray) and v.ndim == 3 and v.shape[1] == prof["nlay"]:
            f[k] = np.ascontiguousarray(v[:, ::-1])
    return f


def _rel(a, b, floor=0.0):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def _both(gpu, osw, prof, flags=None, **opt):
    ref = sw.alloc_outputs(prof["npts"], prof["nlay"], **opt)
    rc, msg = osw.run(prof, ref, flags=flags)
    assert rc == 0, msg
    out = sw.alloc_outputs(prof["npts"], prof["nlay"], **opt)
    gpu.rrtmg_sw_run(prof, out, flags=flags)
    return out, ref


def _check(out, ref):
    for k in ("topflx", "sfcflx", "fdncmp", "flxprf"):
        if k in out:
            assert np.isfinite(out[k]).all(), k
            assert _rel(out[k], ref[k], 1e-300) <= FLUX_RTOL, (k, _rel(out[k], ref[k], 1e-300))
    for k in ("hswc", "hsw0", "hswb"):
        if k in out:
            assert _rel(out[k], ref[k], 1.0) <= HR_TOL, (k, _rel(out[k], ref[k], 1.0))
    assert _rel(out["cldtau"], ref["cldtau"], 1.0) <= 1e-14


def test_sw_allsky_127(gpu, osw):
    prof = _profile(96, 127, 21, night_fraction=0.2, precip=True)
    out, ref = _both(gpu, osw, prof, hswb=True, flxprf=True)
    _check(out, ref)
    assert (ref["topflx"][:, 0] != ref["topflx"][:, 2]).any()   # cloudy columns present


@pytest.mark.parametrize("iovr,isubcsw", [(1, 2), (3, 2), (5, 2), (1, 0)])
def test_sw_top_at_1(gpu, osw, iovr, isubcsw):
    prof = _profile(40, 64, 22, precip=True)
    out, ref = _both(gpu, osw, _flip(prof), flags=dict(top_at_1=1, iovr=iovr, isubcsw=isubcsw), hswb=True,
                     flxprf=True)
    _check(out, ref)


def test_sw_grid_mean_without_seeds(gpu, osw):
    """isubcsw=0 draws no sub-columns: icseed may be absent."""
    prof = _profile(24, 50, 30, precip=True)
    prof["icseed"] = None
    ref = sw.alloc_outputs(24, 50, flxprf=True)
    rc, msg = osw.run(prof, ref, flags=dict(isubcsw=0))
    assert rc == 0, msg
    out = sw.alloc_outputs(24, 50, flxprf=True)
    gpu.rrtmg_sw_run(prof, out, flags=dict(isubcsw=0))
    _check(out, ref)


@pytest.mark.parametrize("flags", [
    dict(iovr=0), dict(iovr=2), dict(iovr=3), dict(iovr=4), dict(iovr=5), dict(iswmode=1), dict(iswmode=3), dict(iswcice=1), dict(iswcice=2),
    dict(iswcliq=2), dict(isubcsw=1), dict(inc_minor_gas=0), dict(isubcsw=0), dict(isubcsw=0, iovr=0),
    dict(isubcsw=0, iswmode=3),
])
def test_sw_options(gpu, osw, flags):
    prof = _profile(48, 72, 23, night_fraction=0.1, precip=True)
    out, ref = _both(gpu, osw, prof, flags=flags, flxprf=True)
    _check(out, ref)


def test_sw_diagnostic_clouds(gpu, osw):
    prof = _profile(32, 50, 24)
    cf = prof["cld_cf"]
    rng = np.random.default_rng(3)
    prof["cld_od"] = np.where(cf > 0, rng.uniform(0.5, 30, cf.shape), 0.0)
    prof["cld_ssa"] = rng.uniform(0.9, 1.0, cf.shape)
    prof["cld_asy"] = rng.uniform(0.7, 0.9, cf.shape)
    out, ref = _both(gpu, osw, prof, flags=dict(iswcliq=0), hswb=True)
    _check(out, ref)


def test_sw_clear_and_one_column(gpu, osw):
    prof = _profile(20, 40, 25, cloudy=False, aerosol=False)
    out, ref = _both(gpu, osw, prof, flxprf=True)
    _check(out, ref)
    prof = _profile(1, 127, 26)
    out, ref = _both(gpu, osw, prof)
    _check(out, ref)


def test_sw_device_memory(gpu, osw):
    import torch
    prof = _profile(64, 127, 27, night_fraction=0.3, precip=True)
    ref = sw.alloc_outputs(64, 127, hswb=True, flxprf=True)
    assert osw.run(prof, ref)[0] == 0
    dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in prof.items()}
    like = torch.zeros(1, device="cuda")
    out = sw.alloc_outputs(64, 127, hswb=True, flxprf=True, like=like)
    kms = [0.0, 0.0, 0.0]
    gpu.rrtmg_sw_run(dev, out, device_memory=True, kernel_ms=kms)
    torch.cuda.synchronize()
    _check({k: v.cpu().numpy() for k, v in out.items()}, ref)
    assert all(t > 0 for t in kms)


def test_sw_gas_optics_stage(gpu, osw):
    """taug, taur, sfluxzen of the optics kernel against setcoef + taumol."""
    import ctypes as C
    import torch
    prof = _profile(12, 90, 28, night_fraction=0.3)
    nday, nl = len(prof["idxday"]), 90
    keep = []
    dev = {k: torch.as_tensor(np.ascontiguousarray(v)).cuda() for k, v in prof.items() if isinstance(v, np.ndarray)}
    ad = sw.make_run_args(dict(prof, **dev), sw.alloc_outputs(12, nl, like=dev["plyr"]), keep=keep)
    tg = torch.zeros(nday, nl, 112, dtype=torch.float64, device="cuda")
    tr, sf = torch.zeros_like(tg), torch.zeros(nday, 112, dtype=torch.float64, device="cuda")
    msg = C.create_string_buffer(256)
    rc = sw.lib().rrtmg_sw_gpu_gas_optics(C.byref(ad), tg.data_ptr(), tr.data_ptr(), sf.data_ptr(), None, msg, 256)
    assert rc == 0, msg.value
    for p in range(nday):
        g0, r0, s0, _ = osw.gas_optics(prof, p + 1)
        assert _rel(tg[p].cpu().numpy(), g0, 1e-300) <= 1e-13
        assert _rel(tr[p].cpu().numpy(), r0, 1e-300) <= 1e-13
        assert np.array_equal(sf[p].cpu().numpy(), s0)


def test_sw_refusals_and_noops(gpu):
    prof = _profile(4, 20, 29)
    for flags, word in ((dict(isubcsw=3), "isubcsw=3"), (dict(iovr=6), "iovr=6")):
        with pytest.raises(sw.RrtmgSwError, match=word):
            gpu.rrtmg_sw_run(prof, sw.alloc_outputs(4, 20), flags=flags)
    out = sw.alloc_outputs(4, 20)
    out["hswc"][:] = 7.0
    gpu.rrtmg_sw_run(prof, out, flags=dict(lsswr=0))     # radsw_main.F90:785: no-op
    assert (out["hswc"] == 7.0).all()
    p2 = dict(prof, idxday=np.array([1, 9], np.int32))
    with pytest.raises(sw.RrtmgSwError, match="idxday"):
        gpu.rrtmg_sw_run(p2, sw.alloc_outputs(4, 20))


@pytest.mark.parametrize("name", ["sw_allsky_127lay", "sw_dcorr_127lay", "sw_gridmean_64lay"])
def test_sw_golden_fixture(gpu, name):
    """The CUDA path against the committed outputs of the restatement."""
    import importlib.util
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "make_sw_golden.py")
    spec = importlib.util.spec_from_file_location("make_sw_golden", path)
    g = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(g)
    case = g.CASES[name]
    prof = g.profile(case)
    out = sw.alloc_outputs(case["npts"], case["nlay"], hswb=True, flxprf=True)
    gpu.rrtmg_sw_run(prof, out, flags=case["flags"])
    ref = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"oracle_{name}.npz")))
    _check(out, ref)


def test_sw_edges(gpu, osw):
    """200 layers (the most this path takes), 2 layers, idxday in arbitrary
    order, and no daytime point at all (radsw_main.F90:786: outputs untouched)."""
    for npts, nlay in ((12, 200), (16, 2), (10, 1)):
        prof = _profile(npts, nlay, 31, night_fraction=0.3, precip=True)
        out, ref = _both(gpu, osw, prof, hswb=True, flxprf=True)
        _check(out, ref)
    prof = _profile(30, 60, 32, night_fraction=0.2)
    prof["idxday"] = np.random.default_rng(5).permutation(prof["idxday"]).astype(np.int32)
    out, ref = _both(gpu, osw, prof, flxprf=True)
    _check(out, ref)
    prof["idxday"] = np.zeros(0, np.int32)
    out = sw.alloc_outputs(30, 60)
    out["hswc"][:] = 5.0
    gpu.rrtmg_sw_run(prof, out)
    assert (out["hswc"] == 5.0).all()


def test_sw_leading_dimension(gpu, osw):
    """Arrays that are (ldim, ...) slices with ldim > npts, host and device memory."""
    import torch
    npts, ld, nlay = 20, 27, 48
    big = _profile(ld, nlay, 33, night_fraction=0.25, precip=True)
    prof = dict(big, npts=npts)
    prof["idxday"] = big["idxday"][big["idxday"] <= npts].astype(np.int32)
    ref = sw.alloc_outputs(ld, nlay, flxprf=True)
    rc, msg = osw.run(prof, ref, flags=None, ldim=ld)
    assert rc == 0, msg
    out = sw.alloc_outputs(ld, nlay, flxprf=True)
    gpu.rrtmg_sw_run(prof, out, ldim=ld)
    _check({k: v for k, v in out.items()}, ref)
    dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in prof.items()}
    outd = sw.alloc_outputs(ld, nlay, flxprf=True, like=dev["plyr"])
    gpu.rrtmg_sw_run(dev, outd, device_memory=True, ldim=ld)
    _check({k: v.cpu().numpy() for k, v in outd.items()}, ref)


def test_sw_host_pipeline(gpu, osw):
    """Host arrays of >= 8,192 columns take the chunked, double-buffered copy
    path: same results as the device-resident call, isubcsw = 1 seeds global,
    daytime points in arbitrary order, and a leading dimension above npts."""
    import torch
    npts, ld, nlay = 9000, 9011, 40
    big = _profile(ld, nlay, 34, night_fraction=0.4, precip=True)
    prof = dict(big, npts=npts)
    prof["idxday"] = np.random.default_rng(7).permutation(big["idxday"][big["idxday"] <= npts]).astype(np.int32)
    for flags in (None, dict(isubcsw=1)):
        out = sw.alloc_outputs(ld, nlay, hswb=True, flxprf=True)
        gpu.rrtmg_sw_run(prof, out, flags=flags, ldim=ld)
        dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
               for k, v in prof.items()}
        outd = sw.alloc_outputs(ld, nlay, hswb=True, flxprf=True, like=dev["plyr"])
        gpu.rrtmg_sw_run(dev, outd, flags=flags, device_memory=True, ldim=ld)
        for k, v in outd.items():
            assert np.array_equal(out[k], v.cpu().numpy()), k
    # and the oracle on a sample of those columns
    sel = prof["idxday"][:64]
    sub = dict(prof, idxday=sel.astype(np.int32))
    ref = sw.alloc_outputs(ld, nlay, flxprf=True)
    assert osw.run(sub, ref, flags=dict(isubcsw=1), ldim=ld)[0] == 0
    cols = sel - 1
    for k in ("topflx", "sfcflx"):
        assert _rel(out[k][cols], ref[k][cols], 1e-300) <= FLUX_RTOL, k


@pytest.mark.parametrize("nlay", [1, 33, 127, 200])
@pytest.mark.parametrize("iovr", [0, 1, 2, 3, 4, 5])
def test_sw_mcica_bits_exact(gpu, osw, nlay, iovr):
    """rrtmg_sw_gpu_mcica against the restatement's mcica_subcol, bit for bit:
    seeds 0 (-> 4357), negative and 2^31-1, cloud fractions of exactly 0, 1
    and 0.5 beside random ones, and fractions under 1e-12 floored to 0."""
    import ctypes as C
    import torch
    n = 24
    rng = np.random.default_rng(nlay * 10 + iovr)
    cf = rng.uniform(0, 1, (nlay, n)) * (rng.uniform(0, 1, (nlay, n)) > 0.4)
    cf[::7] = 1.0
    cf[3::11] = 0.5
    cf[5::13] = 3e-13
    cldf = np.where(cf < 1e-12, 0.0, cf)
    seed = rng.integers(-2**31, 2**31 - 1, n).astype(np.int32)
    seed[:3] = (0, -1, 2**31 - 1)
    dz = rng.uniform(0.05, 1.5, (nlay, n))
    dl = rng.uniform(0.5, 4.0, n)
    alpha = rng.uniform(0, 1, (nlay, n))
    nw = (nlay + 31) // 32
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a)).cuda()
    d_seed, d_cf, d_dz, d_dl, d_al = t(seed), t(cldf), t(dz), t(dl), t(alpha)
    bits = torch.zeros(n * 112 * nw, dtype=torch.int32, device="cuda")
    msg = C.create_string_buffer(256)
    rc = sw.lib().rrtmg_sw_gpu_mcica(n, nlay, 0, iovr, d_seed.data_ptr(), d_cf.data_ptr(), d_dz.data_ptr(),
                                     d_dl.data_ptr(), d_al.data_ptr(), bits.data_ptr(), None, msg, 256)
    assert rc == 0, msg.value
    got = bits.cpu().numpy().view(np.uint32).reshape(n, 112, nw)
    for c in range(n):
        want = osw.mcica_bits(nlay, int(seed[c]), iovr, cldf[:, c], dz=dz[:, c], de_lgth=float(dl[c]),
                              alpha=alpha[:, c])
        assert np.array_equal(got[c], want), (c, iovr)


@pytest.mark.parametrize("flags", [None, dict(iovr=3), dict(isubcsw=0), dict(isubcsw=1)])
def test_sw_run_blocks_equals_per_block_calls(gpu, flags):
    """rrtmg_sw_gpu_run_blocks over uneven physics blocks (one with ldim >
    npts, one without a daytime point) gives, bit for bit, what one call per
    block gives."""
    import torch
    sizes = [5, 37, 1, 64, 12, 9, 130]
    nlay = 50
    profs, ldims = [], []
    off = 0
    for b, n in enumerate(sizes):
        ld = n + (3 if b == 3 else 0)
        p = sw.add_sw_inputs(synthetic.make_profiles(ld, nlay, seed=50, col_offset=off), seed=50, col_offset=off,
                             night_fraction=1.0 if b == 4 else 0.3, precip=True)
        p["npts"] = n
        p["idxday"] = p["idxday"][p["idxday"] <= n].astype(np.int32)
        profs.append({k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
                      for k, v in p.items()})
        ldims.append(ld if ld != n else 0)
        off += ld
    assert len(profs[4]["idxday"]) == 0
    like = profs[0]["plyr"]
    outs_b = [sw.alloc_outputs(ldims[b] or n, nlay, hswb=True, flxprf=True, like=like) for b, n in enumerate(sizes)]
    outs_1 = [sw.alloc_outputs(ldims[b] or n, nlay, hswb=True, flxprf=True, like=like) for b, n in enumerate(sizes)]
    for o in outs_b + outs_1:
        o["hswc"].fill_(7.0)   # the block without a daytime point keeps this
    sw.rrtmg_sw_run_blocks(profs, outs_b, flags=flags, ldims=ldims)
    for b in range(len(sizes)):
        gpu.rrtmg_sw_run(profs[b], outs_1[b], flags=flags, device_memory=True, ldim=ldims[b])
    for b in range(len(sizes)):
        for k in outs_b[b]:
            assert torch.equal(outs_b[b][k], outs_1[b][k]), (b, k)
    assert (outs_b[4]["hswc"] == 7.0).all()


# ---- rrtmg_sw_post_run (rrtmg_sw_post.F90:13-129): bit-exact

_POST_OUT = ("nirbmdi", "nirdfdi", "visbmdi", "visdfdi", "nirbmui", "nirdfui", "visbmui", "visdfui", "sfcdsw",
             "sfcnsw", "htrsw", "swhc", "scmpsw", "sfcfsw", "topfsw")


def _post_arrays(rng, im, levs, ltp, lm):
    ins = dict(sfcalb1=rng.uniform(0, 1, im), sfcalb2=rng.uniform(0, 1, im), sfcalb3=rng.uniform(0, 1, im),
               sfcalb4=rng.uniform(0, 1, im), htswc=rng.normal(size=(lm + ltp, im)),
               htsw0=rng.normal(size=(lm + ltp, im)))
    outs = {n: np.full(im, 7.0) for n in _POST_OUT[:10]}
    outs.update(htrsw=np.full((levs, im), 7.0), swhc=np.full((levs, im), 7.0),
                scmpsw=rng.uniform(0, 500, (im, 6)), sfcfsw=rng.uniform(0, 900, (im, 4)),
                topfsw=rng.uniform(0, 1300, (im, 3)))
    return ins, outs


@pytest.mark.parametrize("device", [True, False])
@pytest.mark.parametrize("nday,lm,ltp,kd,levs,swhtr", [(3, 127, 0, 0, 127, True), (5, 64, 1, 1, 70, True),
                                                       (2, 64, 1, 0, 64, False), (0, 127, 0, 0, 127, True),
                                                       (0, 64, 1, 1, 70, False)])
def test_sw_post_matches_oracle(gpu, osw, device, nday, lm, ltp, kd, levs, swhtr):
    import torch
    from ccpp_physics_b200.rrtmg_sw_post import rrtmg_sw_post_run
    rng = np.random.default_rng(lm + levs + nday)
    im = 1500
    ins, outs = _post_arrays(rng, im, levs, ltp, lm)
    ref = {k: v.copy() for k, v in outs.items()}
    osw.post(im, lm, levs, ltp, nday, lm, kd, True, swhtr, *ins.values(), *ref.values())
    if device:
        ins = {k: torch.from_numpy(v).cuda() for k, v in ins.items()}
        outs = {k: torch.from_numpy(v).cuda() for k, v in outs.items()}
    msg, err = rrtmg_sw_post_run(im, lm, levs, ltp, nday, lm, kd, True, swhtr, *ins.values(), *outs.values())
    assert err == 0, msg
    for k in _POST_OUT:
        g = outs[k].cpu().numpy() if device else outs[k]
        assert np.array_equal(g, ref[k]), k


def test_sw_chain_run_post_on_device(gpu, osw):
    """rrtmg_sw_run -> rrtmg_sw_post_run with every array on the device: the
    post step moves the run's values bit for bit, and the chain meets the run's
    bars against the same chain in the oracle."""
    import torch
    from ccpp_physics_b200.rrtmg_sw_post import rrtmg_sw_post_run
    npts, nlay = 96, 127
    prof = _profile(npts, nlay, 33, night_fraction=0.25, precip=True)
    nday = len(prof["idxday"])
    ref = sw.alloc_outputs(npts, nlay)
    assert osw.run(prof, ref)[0] == 0
    dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in prof.items()}
    out = sw.alloc_outputs(npts, nlay, like=torch.zeros(1, device="cuda"))
    gpu.rrtmg_sw_run(dev, out, device_memory=True)
    alb = [prof[n] for n in ("sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir", "sfcalb_uvis_dif")]

    def post_outs(z):
        o = {n: z(npts) for n in _POST_OUT[:10]}
        o.update(htrsw=z(nlay, npts), swhc=z(nlay, npts))
        return o

    po = post_outs(lambda *s: torch.full(s, 7.0, dtype=torch.float64, device="cuda"))
    msg, err = rrtmg_sw_post_run(npts, nlay, nlay, 0, nday, nlay, 0, True, True, *[dev[n] for n in (
        "sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir", "sfcalb_uvis_dif")], out["hswc"], out["hsw0"],
        *po.values(), out["fdncmp"], out["sfcflx"], out["topflx"])
    assert err == 0, msg
    got = {k: v.cpu().numpy() for k, v in po.items()}
    run = {k: v.cpu().numpy() for k, v in out.items()}
    moved = post_outs(lambda *s: np.full(s, 7.0))
    osw.post(npts, nlay, nlay, 0, nday, nlay, 0, True, True, *alb, run["hswc"], run["hsw0"], *moved.values(),
             run["fdncmp"], run["sfcflx"], run["topflx"])
    for k in got:
        assert np.array_equal(got[k], moved[k]), k
    chain = post_outs(lambda *s: np.full(s, 7.0))
    osw.post(npts, nlay, nlay, 0, nday, nlay, 0, True, True, *alb, ref["hswc"], ref["hsw0"], *chain.values(),
             ref["fdncmp"], ref["sfcflx"], ref["topflx"])
    for k in got:
        floor = 1.0 if k in ("htrsw", "swhc") else 1e-300
        tol = HR_TOL if k in ("htrsw", "swhc") else FLUX_RTOL
        if k == "sfcnsw":
            # a difference of two fluxes: the bar is relative to the downward flux
            assert np.max(np.abs(got[k] - chain[k]) / np.maximum(chain["sfcdsw"], 1e-300)) <= 2 * FLUX_RTOL
        else:
            assert _rel(got[k], chain[k], floor) <= tol, (k, _rel(got[k], chain[k], floor))


# ---- rad_sw_pre_run (rad_sw_pre.F90:14-51): bit-exact

@pytest.mark.parametrize("device", [True, False])
@pytest.mark.parametrize("im", [1, 31, 1024, 1025, 5000, 884_736])
def test_sw_pre_matches_oracle(gpu, osw, device, im):
    import torch
    from ccpp_physics_b200.rad_sw_pre import rad_sw_pre_run
    rng = np.random.default_rng(im)
    cz = rng.uniform(-1, 1, im)
    cz[::7] = 1e-4
    cz[1::11] = np.nextafter(1e-4, 0)
    cz[2::13] = np.nextafter(1e-4, 1)
    for lsswr in (True, False):
        nref, iref = osw.pre(im, lsswr, cz)
        idx = np.full(im, 9, np.int32)
        czg = cz
        if device:
            idx, czg = torch.from_numpy(idx).cuda(), torch.from_numpy(cz).cuda()
        nday, msg, err = rad_sw_pre_run(im, lsswr, czg, idx)
        assert err == 0, msg
        got = idx.cpu().numpy() if device else idx
        assert nday == nref and np.array_equal(got, iref), (lsswr, nday, nref)


def test_sw_chain_pre_run_post_on_device(gpu, osw):
    """rad_sw_pre_run -> rrtmg_sw_run -> rrtmg_sw_post_run, every array on the
    device, against the same chain in the oracle."""
    import torch
    from ccpp_physics_b200.rad_sw_pre import rad_sw_pre_run
    from ccpp_physics_b200.rrtmg_sw_post import rrtmg_sw_post_run
    npts, nlay = 200, 127
    prof = _profile(npts, nlay, 41, night_fraction=0.4, precip=True)
    night = np.ones(npts, bool)
    night[prof["idxday"] - 1] = False
    coszen = np.where(night, -0.3, prof["cosz"])
    nref, iref = osw.pre(npts, True, coszen)
    assert nref == len(prof["idxday"]) and np.array_equal(iref[:nref], prof["idxday"])
    ref = sw.alloc_outputs(npts, nlay)
    assert osw.run(dict(prof, idxday=iref[:nref].copy()), ref)[0] == 0

    dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in prof.items()}
    idx = torch.zeros(npts, dtype=torch.int32, device="cuda")
    nday, msg, err = rad_sw_pre_run(npts, True, torch.from_numpy(coszen).cuda(), idx)
    assert err == 0 and nday == nref, msg
    dev["idxday"] = idx[:nday]
    out = sw.alloc_outputs(npts, nlay, like=torch.zeros(1, device="cuda"))
    gpu.rrtmg_sw_run(dev, out, device_memory=True)
    _check({k: v.cpu().numpy() for k, v in out.items()}, ref)

    names = ("sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir", "sfcalb_uvis_dif")
    po = {n: torch.zeros(npts, dtype=torch.float64, device="cuda") for n in _POST_OUT[:10]}
    po.update(htrsw=torch.zeros((nlay, npts), dtype=torch.float64, device="cuda"),
              swhc=torch.zeros((nlay, npts), dtype=torch.float64, device="cuda"))
    msg, err = rrtmg_sw_post_run(npts, nlay, nlay, 0, nday, nlay, 0, True, True, *[dev[n] for n in names],
                                 out["hswc"], out["hsw0"], *po.values(), out["fdncmp"], out["sfcflx"],
                                 out["topflx"])
    assert err == 0, msg
    pr = {n: np.zeros(npts) for n in _POST_OUT[:10]}
    pr.update(htrsw=np.zeros((nlay, npts)), swhc=np.zeros((nlay, npts)))
    osw.post(npts, nlay, nlay, 0, nref, nlay, 0, True, True, *[prof[n] for n in names], ref["hswc"], ref["hsw0"],
             *pr.values(), ref["fdncmp"], ref["sfcflx"], ref["topflx"])
    for k, v in po.items():
        g = v.cpu().numpy()
        if k in ("htrsw", "swhc"):
            assert _rel(g, pr[k], 1.0) <= HR_TOL, k
        elif k == "sfcnsw":
            assert np.max(np.abs(g - pr[k]) / np.maximum(pr["sfcdsw"], 1e-300)) <= 2 * FLUX_RTOL
        else:
            assert _rel(g, pr[k], 1e-300) <= FLUX_RTOL, k
