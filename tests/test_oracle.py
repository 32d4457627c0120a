"""CPU tests of the restatement oracle and the coefficient tables.

The reference ships no tests or golden vectors for this path (its CI only
checks ASCII encoding), so the pins here are: literals read from the DATA
text of radlw_datatb.f, numpy's independent MT19937 for the twister core,
closed-form checks of the rlwinit tables, and regression fixtures.
"""
import json
import os

import numpy as np
import pytest

from ccpp_physics_b200 import synthetic

GOLD = os.path.join(os.path.dirname(__file__), "golden")
DATA = os.path.join(os.path.dirname(__file__), "..", "ccpp_physics_b200", "data")


def _blob():
    man = json.load(open(os.path.join(DATA, "rrtmg_lw_tables.json")))
    return man, np.fromfile(os.path.join(DATA, "rrtmg_lw_tables.bin"), "<f8")


def _fortran_linear(section, shape):
    """Linear index (0-based) of the first and last element of a DATA section."""
    subs = [s.strip() for s in section.split(",")] if section else [":"] * len(shape)
    firsts, lasts = [], []
    for s, n in zip(subs, shape):
        if s == ":":
            firsts.append(1); lasts.append(n)
        elif ":" in s:
            a, b = s.split(":"); firsts.append(int(a)); lasts.append(int(b))
        else:
            firsts.append(int(s)); lasts.append(int(s))
    def lin(ix):
        l, st = 0, 1
        for i, n in zip(ix, shape):
            l += (i - 1) * st; st *= n
        return l
    return lin(firsts), lin(lasts)


def test_table_blob_checksum_and_literals():
    import hashlib
    man, blob = _blob()
    assert hashlib.sha256(blob.tobytes()).hexdigest() == man["sha256"]
    lits = json.load(open(os.path.join(GOLD, "dtb_literals.json")))
    by_name = {(a["module"], a["name"]): (c, a) for c, a in man["arrays"].items()}
    checked = 0
    for L in lits:
        key = (L["module"], L["name"])
        if key not in by_name:
            continue            # arrays the LW path does not read (none today)
        cname, a = by_name[key]
        i0, i1 = _fortran_linear(L["section"], a["shape"])
        assert blob[a["offset"] + i0] == float(L["first"].lower().replace("d", "e")), (cname, L)
        assert blob[a["offset"] + i1] == float(L["last"].lower().replace("d", "e")), (cname, L)
        checked += 1
    assert checked >= 120
    # known anchors: totplnk(1,1) (radlw_datatb.f:79-80) and preflog(1) (:775-776)
    assert blob[man["arrays"]["totplnk"]["offset"]] == 0.14783e-05
    assert blob[man["arrays"]["preflog"]["offset"]] == 6.96


def test_mt_core_matches_numpy(oracle_lib):
    for seed in (0, 1, 141, 2**31 - 1, -5, 987654):
        u, x, st = oracle_lib.mt_stream(seed, 3000)
        bg = np.random.MT19937()
        bg.state = {"bit_generator": "MT19937", "state": {"key": st.copy(), "pos": 624}}
        assert np.array_equal(u, bg.random_raw(3000).astype(np.uint32))
        s0 = 4357 if seed == 0 else seed & 0xFFFFFFFF
        assert int(st[0]) == s0
        assert all(int(st[i]) == (69069 * int(st[i - 1])) & 0xFFFFFFFF for i in range(1, 624))
        assert np.array_equal(x, u.astype(np.float64) / 4294967295.0)


def test_mt_fixture(oracle_lib):
    gold = json.load(open(os.path.join(GOLD, "mt_words.json")))
    for seed, g in gold.items():
        u, x, _ = oracle_lib.mt_stream(int(seed), 1300)
        got = [int(v) for v in u[:8]] + [int(u[623]), int(u[624]), int(u[1299])]
        assert got == g["u32"]
        assert [float(v) for v in x[:8]] == g["real"]


def test_rlwinit_tables(oracle_lib):
    tau, ex, tfn, fh = oracle_lib.tables()
    bpade = 1.0 / 0.278
    i = np.arange(1, 10000)
    assert tau[0] == 0 and ex[0] == 1 and tfn[0] == 0
    assert tau[10000] == 1e10 and ex[10000] == 1e-20 and tfn[10000] == 1
    assert np.array_equal(tau[1:10000], bpade * (i / (10000 - i)))
    lim = tau[1:10000] >= 708.0                          # aint(-log(tiny(1d0)))
    assert np.all(ex[1:10000][lim] == 1e-20)
    assert np.allclose(ex[1:10000][~lim], np.exp(-tau[1:10000][~lim]), rtol=1e-15, atol=0)
    small = tau[1:10000] < 0.06
    assert np.array_equal(tfn[1:10000][small], tau[1:10000][small] / 6.0)
    assert fh[0] == np.pi * 2e4
    assert fh[1] == 9.80665 * 864.0 / 1.0046e3


@pytest.mark.parametrize("name", ["c1_clear_64lay", "c2_allsky_127lay"])
def test_oracle_regression(oracle_lib, name):
    g = np.load(os.path.join(GOLD, f"oracle_{name}.npz"))
    cfg = json.loads(str(g["cfg"]))
    prof = synthetic.make_profiles(cfg["npts"], cfg["nlay"], seed=cfg["seed"], cloudy=cfg["cloudy"])
    rc, msg, out = oracle_lib.rrtmg_lw_run(prof, hlw0=True, hlwb=True, flxprf=True, nthreads=2)
    assert rc == 0, msg
    for k in ("hlwc", "hlw0", "hlwb", "topflx", "sfcflx", "cldtau", "flxprf"):
        assert np.array_equal(out[k], g[k]), k


def test_physical_sanity(oracle_lib):
    prof = synthetic.make_profiles(32, 127, seed=3)
    rc, msg, out = oracle_lib.rrtmg_lw_run(prof, flxprf=True)
    assert rc == 0, msg
    olr = out["topflx"][:, 0]
    assert np.all((olr > 80) & (olr < 340))
    assert np.all(out["sfcflx"][:, 2] > 100)           # downward LW at the surface
    # clear-sky OLR is never below all-sky OLR for these cold-topped clouds
    assert np.all(out["topflx"][:, 1] >= out["topflx"][:, 0] - 1e-9)
    # flux profile endpoints equal the surface/top records
    fp = out["flxprf"]
    assert np.array_equal(fp[0, :, 0], out["sfcflx"][:, 0])
    assert np.array_equal(fp[-1, :, 0], out["topflx"][:, 0])
    # heating rate = g/cp * dFnet/dp (K/day), recomputed from the profile
    fnet = fp[:, :, 0] - fp[:, :, 1]
    hr = (fnet[:-1] - fnet[1:]) * (9.80665 * 864.0 / 1.0046e3) / prof["delpin"]
    assert np.allclose(hr, out["hlwc"], rtol=1e-12, atol=1e-12)


def test_top_at_1_is_a_flip(oracle_lib):
    prof = synthetic.make_profiles(8, 40, seed=5)
    rc, _, ref = oracle_lib.rrtmg_lw_run(prof, hlwb=True, flxprf=True)
    flip = dict(prof)
    for k, v in prof.items():
        if isinstance(v, np.ndarray) and v.ndim >= 2 and k not in ("alpha",):
            flip[k] = np.ascontiguousarray(v[..., ::-1, :]) if v.ndim == 3 else np.ascontiguousarray(v[::-1])
    rc, msg, out = oracle_lib.rrtmg_lw_run(flip, flags={"top_at_1": 1}, hlwb=True, flxprf=True)
    assert rc == 0, msg
    assert np.array_equal(out["topflx"], ref["topflx"])
    assert np.array_equal(out["sfcflx"], ref["sfcflx"])
    assert np.array_equal(out["hlwc"][::-1], ref["hlwc"])
    assert np.array_equal(out["cldtau"][::-1], ref["cldtau"])
    assert np.array_equal(out["hlwb"][:, ::-1], ref["hlwb"])
    assert np.array_equal(out["flxprf"][::-1], ref["flxprf"])


def test_error_paths(oracle_lib):
    prof = synthetic.make_profiles(4, 20, seed=1)
    p2 = dict(prof)
    p2["cld_swp"] = None
    rc, msg, _ = oracle_lib.rrtmg_lw_run(p2)
    assert rc == 1 and msg.startswith("Logic error: ilwcliq>0 requires")
    rc, msg, _ = oracle_lib.rrtmg_lw_run(prof, flags={"ilwcliq": 0})
    assert rc == 1 and "cld_od" in msg
    out = None
    rc, msg, out = oracle_lib.rrtmg_lw_run(prof, flags={"lslwr": 0})
    assert rc == 0 and np.isnan(out["hlwc"]).all()     # immediate return, nothing written
    rc, msg = oracle_lib.rlwinit(iovr=9)
    assert rc == 1 and "overlap" in msg
    oracle_lib.rlwinit()


def test_mcica_max_random_properties(oracle_lib):
    rng = np.random.default_rng(0)
    cldf = np.where(rng.random(60) < 0.4, rng.random(60), 0.0)
    cldf[10:14] = 1.0
    lc = oracle_lib.mcica(cldf, 77, iovr=1)
    # fully overcast layers are cloudy in every sub-column, clear layers never
    assert lc[10:14].all()
    assert not lc[cldf == 0].any()
    # cloud fraction is reproduced statistically over 140 sub-columns
    frac = lc.mean(axis=1)
    m = (cldf > 0.2) & (cldf < 0.8)
    assert np.abs(frac[m] - cldf[m]).mean() < 0.12
    # maximum overlap in adjacent cloudy layers: a sub-column cloudy in the
    # layer below stays cloudy above when the upper fraction is not smaller
    for k in range(1, 60):
        if cldf[k] >= cldf[k - 1] > 0:
            assert np.all(lc[k][lc[k - 1]])


def test_mcica_draw_conversion_exhaustive(oracle_lib):
    """The GPU McICA kernel converts each 32-bit draw u to u / (2^32 - 1)
    without a division (one FMA and an exact-tie fix); that must equal the
    reference's division for all 2^32 values of u."""
    import time
    t0 = time.time()
    bad = oracle_lib.lib().oracle_check_u32_unit(0, 1 << 32)
    assert bad == 0
    assert time.time() - t0 < 120


def test_grid_cloud_transfer_properties(oracle_lib):
    """rtrn (random) and rtrnmr (maximum-random), the isubclw=0 transfer: with
    overcast or clear layers only, rtrn gives McICA's fluxes (its sub-columns
    are then all cloudy or all clear, same equations), and rtrnmr agrees to
    the Pade-table quantisation (it takes the cloudy transmittance from the
    total optical depth's table entry, RLM:3193-3202, not trng * exp(-odcld));
    with partial clouds maximum-random overlap gives more OLR than random
    overlap (fewer distinct cloud layers seen from above)."""
    import numpy as np
    prof = synthetic.make_profiles(24, 60, seed=12)
    cf = prof["cld_cf"]
    cf[:] = np.where(cf > 0, 1.0, 0.0)            # overcast or clear layers only
    outs = {}
    for name, flags in (("mc", dict(isubclw=2, iovr=1)), ("rand", dict(isubclw=0, iovr=0)),
                        ("mr", dict(isubclw=0, iovr=1))):
        rc, msg, o = oracle_lib.rrtmg_lw_run(prof, flags=flags, hlw0=True, hlwb=True)
        assert rc == 0, msg
        outs[name] = o
    for k in ("topflx", "sfcflx", "hlwc", "hlw0", "hlwb"):
        np.testing.assert_allclose(outs["rand"][k], outs["mc"][k], rtol=1e-12, atol=1e-12, err_msg=k)
        np.testing.assert_allclose(outs["mr"][k], outs["mc"][k], rtol=2e-3, atol=2e-2, err_msg=k)
    prof = synthetic.make_profiles(24, 60, seed=13)
    prof["cld_cf"][:] = np.clip(prof["cld_cf"] * 0.7 + 0.2 * (prof["cld_cf"] > 0), 0, 1)
    rc, msg, r = oracle_lib.rrtmg_lw_run(prof, flags=dict(isubclw=0, iovr=0))
    rc2, msg2, m = oracle_lib.rrtmg_lw_run(prof, flags=dict(isubclw=0, iovr=1))
    assert rc == 0 and rc2 == 0
    assert np.all(np.isfinite(m["topflx"])) and np.all(np.isfinite(m["hlwc"]))
    # (up to the table-vs-exp difference of the two routines' cloudy transmittance)
    assert np.all(m["topflx"][:, 0] >= r["topflx"][:, 0] - 0.01)
    assert np.mean(m["topflx"][:, 0]) > np.mean(r["topflx"][:, 0]) + 0.1
    assert np.array_equal(m["topflx"][:, 1], r["topflx"][:, 1])   # clear-sky parts agree exactly
