"""GPU parity of the steps either side of rrtmg_lw_run (csrc/lw_prep.cu,
csrc/lw_mcica.cu seed stream) against the oracle:

* seeds (GFS_rad_time_vary.fv3.F90:59-84): bit-exact, device and host memory;
* decorrelation length and alpha (radiation_cloud_overlap.F90,
  radiation_clouds.f:837-856): Hogan and the constant length bit-exact; the
  terms with exp within 2 ulp (CUDA's exp and libm's are each within 1 ulp),
  the zero pattern exact;
* rrtmg_lw_post_run (rrtmg_lw_post.F90:13-77): bit-exact;
* the chain seeds -> overlap parameters -> rrtmg_lw_run (iovr 3, 4, 5) ->
  post on the device against the same chain in the oracle.
"""
import math

import numpy as np
import pytest

from ccpp_physics_b200 import abi, synthetic

pytestmark = pytest.mark.gpu

FLUX_RTOL = 1e-10


@pytest.fixture(scope="module")
def mods():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ccpp_physics_b200 import cloud_overlap, rad_time_vary, rrtmg_lw, rrtmg_lw_post
    rc, msg = rrtmg_lw.rlwinit(device=0, iovr=3)
    assert rc == 0, msg
    return rrtmg_lw, rad_time_vary, cloud_overlap, rrtmg_lw_post


def _tile(cnx, isc, jsc, nx, ny, seed):
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), indexing="ij")
    o = rng.permutation(nx * ny)
    return i.ravel()[o].astype(np.int32), j.ravel()[o].astype(np.int32)


@pytest.mark.parametrize("cnx,isc,jsc,nx,ny,sec", [(96, 1, 1, 96, 96, 3600.0), (384, 97, 193, 96, 64, 12345.6),
                                                   (7, 3, 2, 5, 6, 0.0)])
@pytest.mark.parametrize("device", [True, False])
def test_seeds_match_oracle(mods, cnx, isc, jsc, nx, ny, sec, device):
    import torch
    from oracle import oracle
    _, rtv, _, _ = mods
    imap, jmap = _tile(cnx, isc, jsc, nx, ny, seed=cnx + nx)
    ipsd0, ipsdlim = 17 * 2026 + 43 * 12 + 37 * 3 + 23 * 0, 100000000
    rc, sw_ref, lw_ref = oracle.seeds(sec=sec, ipsd0=ipsd0, ipsdlim=ipsdlim, cnx=cnx, cny=cnx, isc=isc, jsc=jsc,
                                      imap=imap, jmap=jmap)
    assert rc == 0
    n = imap.size
    if device:
        im, jm = torch.from_numpy(imap).cuda(), torch.from_numpy(jmap).cuda()
        sw, lw = torch.zeros(n, dtype=torch.int32, device="cuda"), torch.zeros(n, dtype=torch.int32, device="cuda")
    else:
        im, jm, sw, lw = imap, jmap, np.zeros(n, np.int32), np.zeros(n, np.int32)
    msg, err = rtv.gfs_rad_time_vary_seeds(False, None, True, True, 2, 2, sw, lw, cnx, cnx, isc, jsc, im, jm, sec,
                                           ipsd0, ipsdlim)
    assert err == 0, msg
    if device:
        sw, lw = sw.cpu().numpy(), lw.cpu().numpy()
    assert np.array_equal(sw, sw_ref) and np.array_equal(lw, lw_ref)


def test_seeds_supplied_skipped_and_bad_index(mods):
    import torch
    _, rtv, _, _ = mods
    n = 300
    rseeds = torch.arange(2 * n, dtype=torch.int32, device="cuda").reshape(2, n) * 3 + 1
    sw, lw = torch.zeros(n, dtype=torch.int32, device="cuda"), torch.zeros(n, dtype=torch.int32, device="cuda")
    ones = torch.ones(n, dtype=torch.int32, device="cuda")
    msg, err = rtv.gfs_rad_time_vary_seeds(True, rseeds, True, False, 2, 0, sw, lw, 4, 4, 1, 1, ones, ones,
                                           60.0, 0, 100)
    assert err == 0, msg
    assert torch.equal(sw, rseeds[0]) and torch.equal(lw, rseeds[1])
    sw.fill_(-1)
    msg, err = rtv.gfs_rad_time_vary_seeds(False, None, True, True, 1, 1, sw, lw, 4, 4, 1, 1, ones, ones, 60.0, 0, 100)
    assert err == 0 and bool((sw == -1).all())
    jbad = ones.clone()
    jbad[17] = 9                          # p beyond the 4 x 4 face: an error, nothing read out of bounds
    msg, err = rtv.gfs_rad_time_vary_seeds(False, None, True, True, 2, 2, sw, lw, 4, 4, 1, 1, ones, jbad, 60.0, 0,
                                           100)
    assert err == 1 and "column 18" in msg


def _ulp_close(got, ref, ulps=2):
    return np.all(np.abs(got - ref) <= ulps * np.spacing(np.abs(ref)))


@pytest.mark.parametrize("iovr", [1, 3, 4, 5])
@pytest.mark.parametrize("idcor", [0, 1, 2])
def test_overlap_params_match_oracle(mods, iovr, idcor):
    import torch
    from oracle import oracle
    _, _, co, _ = mods
    nlay, npts = 127, 2000
    p = synthetic.make_profiles(npts, nlay, seed=41)
    rng = np.random.default_rng(idcor * 10 + iovr)
    lat = rng.uniform(-math.pi / 2, math.pi / 2, npts)
    latdeg = lat * 180.0 / math.pi
    dz, cf = p["dzlyr"], p["cld_cf"]
    jul, yl = 250.5, 365
    dl_ref, al_ref = oracle.overlap_params(iovr, idcor, dz, cf, xlat=lat, latdeg=latdeg, julian=jul, yearlen=yl,
                                           dcorr_con=2.5)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    dl = torch.full((npts,), -1.0, dtype=torch.float64, device="cuda")
    al = torch.full((nlay, npts), -1.0, dtype=torch.float64, device="cuda")
    msg, err = co.overlap_params(iovr, idcor, t(dz), t(cf), dl, al, xlat=t(lat), latdeg=t(latdeg), julian=jul,
                                 yearlen=yl, dcorr_con=2.5)
    assert err == 0, msg
    dl, al = dl.cpu().numpy(), al.cpu().numpy()
    if idcor == 2 and iovr >= 3:
        assert _ulp_close(dl, dl_ref)
    else:
        assert np.array_equal(dl, dl_ref)
    assert np.array_equal(al == 0.0, al_ref == 0.0)
    assert _ulp_close(al, al_ref)


def test_overlap_routines_alone_host_memory(mods):
    from oracle import oracle
    _, _, co, _ = mods
    rng = np.random.default_rng(12)
    npts, nlay = 777, 64
    lat = rng.uniform(-1.5, 1.5, npts)
    d = np.zeros(npts)
    assert co.cmp_dcorr_lgth_hogan(lat, math.pi, d)[1] == 0
    assert np.array_equal(d, oracle.dcorr_hogan(lat))
    latdeg = np.degrees(lat)
    assert co.cmp_dcorr_lgth_oreopoulos(latdeg, 30.0, 366, d)[1] == 0
    assert _ulp_close(d, oracle.dcorr_oreopoulos(latdeg, 30.0, 366))
    dz = rng.uniform(0.02, 2.0, (nlay, npts))
    cf = rng.uniform(0, 1, (nlay, npts)) * (rng.uniform(0, 1, (nlay, npts)) > 0.5)
    al = np.zeros((nlay, npts))
    assert co.get_alpha_exper(5, 5, dz, d, cf, al)[1] == 0
    ref = oracle.alpha_exper(5, 5, dz, d, cf)
    assert np.array_equal(al == 0.0, ref == 0.0) and _ulp_close(al, ref)


@pytest.mark.parametrize("device", [True, False])
@pytest.mark.parametrize("lm,ltp,kd,levs,lwhtr", [(127, 0, 0, 127, True), (64, 1, 1, 70, True),
                                                  (64, 1, 0, 64, False), (5, 0, 0, 9, True)])
def test_post_matches_oracle(mods, device, lm, ltp, kd, levs, lwhtr):
    import torch
    from oracle import oracle
    _, _, _, post = mods
    rng = np.random.default_rng(lm + levs)
    im = 1500
    htlwc, htlw0 = rng.normal(size=(lm + ltp, im)), rng.normal(size=(lm + ltp, im))
    sfc, tsfa = rng.normal(size=(im, 4)), rng.normal(size=im)
    outs_ref = [np.full(im, 7.0), np.full(im, 7.0), np.full((levs, im), 7.0), np.full((levs, im), 7.0)]
    oracle.post(im, levs, ltp, lm, kd, 1, lwhtr, tsfa, htlwc, htlw0, sfc, *outs_ref)
    ins = [tsfa, htlwc, htlw0, sfc]
    outs = [np.full(im, 7.0), np.full(im, 7.0), np.full((levs, im), 7.0), np.full((levs, im), 7.0)]
    if device:
        ins = [torch.from_numpy(a).cuda() for a in ins]
        outs = [torch.from_numpy(a).cuda() for a in outs]
    msg, err = post.rrtmg_lw_post_run(im, levs, ltp, lm, kd, True, lwhtr, *ins, *outs)
    assert err == 0, msg
    for g, r in zip(outs, outs_ref):
        g = g.cpu().numpy() if device else g
        assert np.array_equal(g, r)


@pytest.mark.parametrize("iovr,idcor", [(3, 1), (4, 2), (5, 0)])
def test_chain_seeds_overlap_run_post(mods, oracle_lib, iovr, idcor):
    """seeds -> overlap parameters -> rrtmg_lw_run -> post, all on the device,
    against the same chain in the oracle."""
    import torch
    from oracle import oracle
    lwm, rtv, co, post = mods
    cnx, isc, jsc, nx, ny = 48, 9, 17, 24, 20
    nlay, npts = 127, nx * ny
    imap, jmap = _tile(cnx, isc, jsc, nx, ny, seed=5)
    sec, ipsd0, ipsdlim = 7200.0, 35000, 100000000
    prof = synthetic.make_profiles(npts, nlay, seed=60 + iovr)
    prof["flags"] = dict(prof["flags"], iovr=iovr)
    rng = np.random.default_rng(iovr)
    lat = rng.uniform(-1.5, 1.5, npts)
    latdeg = np.degrees(lat)

    # oracle chain
    _, _, lw_seed = oracle.seeds(sec=sec, ipsd0=ipsd0, ipsdlim=ipsdlim, cnx=cnx, cny=cnx, isc=isc, jsc=jsc,
                                 imap=imap, jmap=jmap)
    dl, al = oracle.overlap_params(iovr, idcor, prof["dzlyr"], prof["cld_cf"], xlat=lat, latdeg=latdeg,
                                   julian=120.0, yearlen=365)
    pr = dict(prof, icseed=lw_seed, de_lgth=dl, alpha=al)
    rc, msg, ref = oracle.rrtmg_lw_run(pr)
    assert rc == 0, msg
    ref_post = [np.zeros(npts), np.zeros(npts), np.zeros((nlay, npts)), np.zeros((nlay, npts))]
    oracle.post(npts, nlay, 0, nlay, 0, 1, 1, prof["tlyr"][0].copy(), ref["hlwc"], ref["hlw0"], ref["sfcflx"],
                *ref_post)

    # device chain
    dprof = lwm.to_device(prof)
    seeds = torch.zeros(npts, dtype=torch.int32, device="cuda")
    sw = torch.zeros_like(seeds)
    msg, err = rtv.gfs_rad_time_vary_seeds(False, None, True, True, 2, 2, sw, seeds, cnx, cnx, isc, jsc,
                                           torch.from_numpy(imap).cuda(), torch.from_numpy(jmap).cuda(), sec, ipsd0,
                                           ipsdlim)
    assert err == 0, msg
    dl_d = torch.zeros(npts, dtype=torch.float64, device="cuda")
    al_d = torch.zeros((nlay, npts), dtype=torch.float64, device="cuda")
    msg, err = co.overlap_params(iovr, idcor, dprof["dzlyr"], dprof["cld_cf"], dl_d, al_d,
                                 xlat=torch.from_numpy(lat).cuda(), latdeg=torch.from_numpy(latdeg).cuda(),
                                 julian=120.0, yearlen=365)
    assert err == 0, msg
    dprof.update(icseed=seeds, de_lgth=dl_d, alpha=al_d)
    o = abi.alloc_outputs(npts, nlay, hlw0=True, like="cuda")
    msg, err = lwm.run_profile(dprof, o)
    assert err == 0, msg
    outs = [torch.zeros(npts, dtype=torch.float64, device="cuda") for _ in range(2)] + \
           [torch.zeros((nlay, npts), dtype=torch.float64, device="cuda") for _ in range(2)]
    msg, err = post.rrtmg_lw_post_run(npts, nlay, 0, nlay, 0, True, True, dprof["tlyr"][0].contiguous(), o["hlwc"],
                                      o["hlw0"], o["sfcflx"], *outs)
    assert err == 0, msg

    assert np.array_equal(seeds.cpu().numpy(), lw_seed)
    for k in ("topflx", "sfcflx"):
        g = o[k].cpu().numpy()
        assert np.max(np.abs(g - ref[k]) / np.maximum(np.abs(ref[k]), 1.0)) < FLUX_RTOL, k
    assert np.max(np.abs(o["hlwc"].cpu().numpy() - ref["hlwc"])) < 1e-9
    # the post step moves the device run's values without touching them
    assert torch.equal(outs[2], o["hlwc"]) and torch.equal(outs[3], o["hlw0"])
    assert torch.equal(outs[1], o["sfcflx"][:, 2].contiguous())
    assert np.max(np.abs(outs[2].cpu().numpy() - ref_post[2])) < 1e-9
