"""CPU tests of the steps either side of rrtmg_lw_run: the oracle's
restatement of the seed preparation (GFS_rad_time_vary.fv3.F90:59-84 with
random_index_t, mersenne_twister.f:489-503), the cloud-overlap parameters
(radiation_cloud_overlap.F90, radiation_clouds.f:837-856) and
rrtmg_lw_post_run (rrtmg_lw_post.F90:13-77), pinned against independent numpy
restatements and closed-form values; and the host-side validation of their
C entry points (no GPU needed for those)."""
import ctypes as C
import math

import numpy as np
import pytest

from ccpp_physics_b200 import abi


def _gfs_stream(seed, m):
    """m raw words of the GFS twister through numpy's own MT19937 core: the
    state is the GFS seeding (mt(0) = seed, 0 -> 4357; mt(i) = 69069 mt(i-1)),
    position 624 so the first draw twists (MT:285-299)."""
    key = np.zeros(624, dtype=np.uint64)
    v = (4357 if seed == 0 else seed) & 0xFFFFFFFF
    for i in range(624):
        key[i] = v
        v = (v * 69069) & 0xFFFFFFFF
    bg = np.random.MT19937(0)
    bg.state = {"bit_generator": "MT19937", "state": {"key": key.astype(np.uint32), "pos": 624}}
    return bg.random_raw(m).astype(np.uint64)


def _numpy_random_index(seed, imax, m):
    h = _gfs_stream(seed, m).astype(np.float64) / 4294967295.0
    return np.maximum(np.ceil(h * imax), 1).astype(np.int32)


@pytest.mark.parametrize("seed,imax", [(1, 100000000), (4357, 7), (0, 1000), (2 ** 31 - 1, 2 ** 31 - 1),
                                       (-5, 12345)])
def test_random_index_matches_numpy_twister(seed, imax):
    from oracle import oracle
    m = 3 * 624 + 17
    got = oracle.random_index(seed, imax, m)
    assert np.array_equal(got, _numpy_random_index(seed, imax, m))
    assert got.min() >= 1 and got.max() <= imax


def _grid_maps(cnx, cny, isc, jsc, nx, ny, rng):
    i, j = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), indexing="ij")
    order = rng.permutation(nx * ny)
    return i.ravel()[order].astype(np.int32), j.ravel()[order].astype(np.int32)


def test_seeds_restatement():
    """numrdm from the numpy twister, picked by the tile's grid indices."""
    from oracle import oracle
    rng = np.random.default_rng(3)
    cnx = cny = 48
    isc, jsc, nx, ny = 13, 25, 24, 16
    imap, jmap = _grid_maps(cnx, cny, isc, jsc, nx, ny, rng)
    sec, ipsd0, ipsdlim = 10800.0, 17 * 2024 + 43 * 7 + 37 * 1 + 23 * 6, 100000000
    rc, sw, lw = oracle.seeds(sec=sec, ipsd0=ipsd0, ipsdlim=ipsdlim, cnx=cnx, cny=cny, isc=isc, jsc=jsc,
                              imap=imap, jmap=jmap)
    assert rc == 0
    ipseed = int(math.floor(100 * math.sqrt(sec) + 0.5)) % ipsdlim + 1 + ipsd0
    numrdm = _numpy_random_index(ipseed, ipsdlim, 2 * cnx * cny)
    p = imap + isc - 1 + (jmap + jsc - 2) * cnx
    assert np.array_equal(sw, numrdm[p - 1])
    assert np.array_equal(lw, numrdm[p - 1 + cnx * cny])


def test_seeds_supplied_and_skipped():
    from oracle import oracle
    n = 20
    rseeds = np.arange(2 * n, dtype=np.int32).reshape(2, n) + 7
    imap = np.ones(n, np.int32)
    rc, sw, lw = oracle.seeds(sec=0.0, ipsd0=0, ipsdlim=10, cnx=4, cny=4, isc=1, jsc=1, imap=imap, jmap=imap,
                              lrseeds=1, rseeds=rseeds)
    assert rc == 0 and np.array_equal(sw, rseeds[0]) and np.array_equal(lw, rseeds[1])
    keep = np.full(n, -3, np.int32)
    rc, sw, lw = oracle.seeds(sec=0.0, ipsd0=0, ipsdlim=10, cnx=4, cny=4, isc=1, jsc=1, imap=imap, jmap=imap,
                              isubc_lw=1, isubc_sw=0, icsdsw=keep.copy(), icsdlw=keep.copy())
    assert rc == 0 and np.all(sw == -3) and np.all(lw == -3)   # GFS_rad_time_vary.fv3.F90:64
    rc, _, _ = oracle.seeds(sec=0.0, ipsd0=0, ipsdlim=10, cnx=4, cny=4, isc=4, jsc=1, imap=imap, jmap=imap * 10)
    assert rc == 1                                              # grid index outside the face


def test_dcorr_known_values():
    from oracle import oracle
    # Hogan et al. (2010) eq. 13: 2.78 at the equator, floor 0.6 from |lat| > 47.0 deg
    lat = np.array([0.0, math.pi / 2, -math.pi / 4, math.pi / 6])
    got = oracle.dcorr_hogan(lat)
    assert got[0] == 2.78 and got[1] == 0.6
    assert got[2] == 2.78 - 4.6 * 0.25 and got[3] == 2.78 - 4.6 * abs(lat[3] / math.pi)
    # Oreopoulos et al. (2012) eqs. 10-11: peak am1 + am2 where lat = am3
    for jul, yl in ((100.0, 365), (200.0, 366), (181.0, 365), (182.0, 365)):
        am3 = (-4 * 7.0 * (jul - 272.0) / yl) if jul > 181.0 else (4 * 7.0 * (jul - 91.0) / yl)
        lats = np.array([am3, am3 + 25.584, -90.0, 90.0])
        d = oracle.dcorr_oreopoulos(lats, jul, yl)
        assert d[0] == 1.4315 + 2.1219
        assert abs(d[1] - (1.4315 + 2.1219 * math.exp(-1.0))) < 1e-15
        ref = 1.4315 + 2.1219 * np.exp(-((lats - am3) ** 2) / (25.584 ** 2))
        assert np.max(np.abs(d - ref)) < 1e-15


def test_alpha_exper_rule():
    from oracle import oracle
    rng = np.random.default_rng(5)
    nlay, ncol = 12, 9
    dz = rng.uniform(0.05, 1.5, (nlay, ncol))
    dl = rng.uniform(0.6, 3.5, ncol)
    cf = rng.uniform(0, 1, (nlay, ncol)) * (rng.uniform(0, 1, (nlay, ncol)) > 0.4)
    a4 = oracle.alpha_exper(4, 5, dz, dl, cf)
    ref = np.exp(-dz / dl)                  # numpy's exp: within one ulp of libm's
    ref[0] = 0.0
    assert np.all(np.abs(a4 - ref) <= np.spacing(ref)) and not a4[0].any()
    a5 = oracle.alpha_exper(5, 5, dz, dl, cf)
    clear_after_cloud = np.zeros_like(cf, bool)
    clear_after_cloud[1:] = (cf[1:] == 0.0) & (cf[:-1] > 0.0)
    assert clear_after_cloud.any()
    assert np.array_equal(a5, np.where(clear_after_cloud, 0.0, a4))


def test_overlap_block():
    from oracle import oracle
    rng = np.random.default_rng(6)
    nlay, ncol = 10, 7
    dz = rng.uniform(0.05, 1.5, (nlay, ncol))
    cf = rng.uniform(0, 1, (nlay, ncol))
    lat = rng.uniform(-1.5, 1.5, ncol)
    dl, al = oracle.overlap_params(1, 1, dz, cf, xlat=lat)          # max-random: both zero
    assert not dl.any() and not al.any()
    dl, al = oracle.overlap_params(4, 0, dz, cf, dcorr_con=2.5)     # constant length
    assert np.all(dl == 2.5) and np.array_equal(al, oracle.alpha_exper(4, 5, dz, dl, cf))
    dl, al = oracle.overlap_params(3, 1, dz, cf, xlat=lat)
    assert np.array_equal(dl, oracle.dcorr_hogan(lat))
    keep = np.full(ncol, 9.0)
    dl, _ = oracle.overlap_params(4, 7, dz, cf, de_lgth=keep)       # no idcor matches: de_lgth kept
    assert np.all(dl == 9.0)


def test_post_restatement():
    from oracle import oracle
    rng = np.random.default_rng(8)
    im, lm, ltp, kd, levs = 11, 6, 1, 1, 9
    htlwc = rng.normal(size=(lm + ltp, im))
    htlw0 = rng.normal(size=(lm + ltp, im))
    sfc = rng.normal(size=(im, 4))
    tsfa = rng.normal(size=im)
    tsflw, sfcdlw = np.zeros(im), np.zeros(im)
    htrlw, lwhc = np.zeros((levs, im)), np.zeros((levs, im))
    oracle.post(im, levs, ltp, lm, kd, 1, 1, tsfa, htlwc, htlw0, sfc, tsflw, sfcdlw, htrlw, lwhc)
    src = np.minimum(np.arange(levs), lm - 1) + kd
    assert np.array_equal(htrlw, htlwc[src]) and np.array_equal(lwhc, htlw0[src])
    assert np.array_equal(tsflw, tsfa) and np.array_equal(sfcdlw, sfc[:, 2])


# ---- host-side validation of the C entry points (returns before any CUDA call)

def _msg():
    return C.create_string_buffer(256)


def test_entry_point_validation():
    from ccpp_physics_b200 import rrtmg_lw as lw
    L = lw.lib()
    x = abi.ExecArgs(memory=abi.HOST, sync=1)
    n = 4
    arr = (C.c_int32 * n)()
    a = abi.SeedArgs(lslwr=1, isubc_lw=2, n=n, ipsdlim=0, cnx=4, cny=4)
    a.imap = a.jmap = a.icsdsw = a.icsdlw = C.cast(arr, C.POINTER(C.c_int32))
    m = _msg()
    assert L.rrtmg_lw_gpu_seeds(C.byref(a), C.byref(x), m, 256) == 1 and b"ipsdlim" in m.value
    a.isubc_lw = 1                        # no McICA seeds wanted: no-op
    assert L.rrtmg_lw_gpu_seeds(C.byref(a), C.byref(x), m, 256) == 0
    o = abi.OverlapArgs(mode=7, npts=3, nlay=2)
    assert L.rrtmg_lw_gpu_overlap_params(C.byref(o), C.byref(x), m, 256) == 1 and b"mode" in m.value
    o = abi.OverlapArgs(mode=abi.OVERLAP_CLOUDS, npts=3, nlay=2, idcor=1, idcor_hogan=1, iovr=4, iovr_exp=4,
                        iovr_dcorr=3, iovr_exprand=5)
    dbl = (C.c_double * 8)()
    o.de_lgth = o.alpha = o.dzlay = C.cast(dbl, C.POINTER(C.c_double))
    assert L.rrtmg_lw_gpu_overlap_params(C.byref(o), C.byref(x), m, 256) == 1 and b"xlat" in m.value
    p = abi.PostArgs(im=2, levs=3, ltp=0, lm=2, kd=1, lslwr=1)
    assert L.rrtmg_lw_gpu_post(C.byref(p), C.byref(x), m, 256) == 1 and b"kd <= ltp" in m.value
    p.lslwr = 0                           # rrtmg_lw_post.F90:41: nothing to do
    assert L.rrtmg_lw_gpu_post(C.byref(p), C.byref(x), m, 256) == 0
