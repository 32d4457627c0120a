"""Benchmark of the B200 RRTMG-LW column path (rrtmg_lw_run replacement).

Workload: 884,736 columns x 127 layers (six 384 x 384 cubed-sphere faces),
all-sky McICA with maximum-random overlap (ilwcliq=1, ilwcice=3, isubclw=2,
seeds = column index), seeded synthetic profiles
(ccpp_physics_b200.synthetic), split into uneven physics blocks of 8..256
columns (sizes U{8..256}, seed 7), each block its own (n_b, nlay) array as a
UFS host allocates them.  One step = one rrtmg_lw_gpu_run_blocks call over
every block of the rank (autotuned launch shape, replayed as a CUDA graph).

The last line printed is the headline JSON record:
  value      plain FP64 path, inputs resident in HBM, columns/s of the job;
  paths      the FP32 and learned-gas-optics paths on the same blocks, with
             their flux / heating-rate RMSE against FP64 and speed-up;
  parity     FP64 GPU outputs against the CPU restatement (oracle/) on the
             first 65,536 columns of the workload and on the 16,384-column
             all-sky case (with flux profiles);
  e2e        the same FP64 work through rrtmg_lw_gpu_run with pinned host
             arrays, host<->device copies inside the timed region;
  roofline   the column kernels against the measured HBM copy bandwidth, and
             fp_pipe their FP64 flops against the measured FMA peak;
  cpu_baseline  the oracle on all host cores, timed on the parity sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--legs sw,callers,train [--only-legs]]
--gpus N > 1 starts N ranks itself (torch.distributed.run) unless it already
runs under a launcher (WORLD_SIZE set).  Each rank takes whole physics blocks
of the workload (ccpp_physics_b200.shard.block_range): the total work is
fixed ("scaling": "strong"), no collective touches the data path, and only
the per-rank times are reduced (max over ranks).  --legs prints the
auxiliary legs (shortwave scheme, the steps either side of the run, the
surrogate's training throughput) as JSON lines before the headline.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import os
import socket
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LW columns/s @127 lev: plain FP64 vs FP32 vs surrogate, flux RMSE vs FP64"
BYTES_PER_COL = 61052     # compulsory HBM bytes per column at 127 layers (FP64 interface)
NCOLS, NLAY = 884_736, 127
WORKLOAD = "c3_physics_blocks_884736x127"
PARITY_SAMPLE = 65_536    # columns of the workload checked against the oracle
C2_COLS = 16_384          # the all-sky McICA case (first columns of the same generator)


def workload_config(world):
    """The `config` object of both arms (identical for the same N)."""
    return {"workload": WORKLOAD, "ncols": NCOLS, "nlay": NLAY,
            "blocks": "U{8..256} (seed 7), 6,686 blocks, each its own (n_b, nlay) array",
            "clouds": "all-sky McICA, max-random overlap (iovr=1, isubclw=2)",
            "parallelism": f"block shards x{world}",
            "l2": "inputs 54 GB per step > 126 MB L2, no flush needed"}


def rank_blocks(rank, world):
    """Physics-block sizes of the workload and this rank's shard of them:
    (all sizes, this rank's sizes, first global column of the shard)."""
    import numpy as np
    from ccpp_physics_b200 import shard, synthetic
    sizes = synthetic.physics_blocks(NCOLS, seed=7)
    b0, b1 = shard.block_range(sizes, rank, world)
    return sizes, sizes[b0:b1], int(np.sum(sizes[:b0]))


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            p = json.load(fh)
        return p.get("hbm_gbs", 6650.0), "measured"
    except OSError:
        return 6650.0, "fallback"


def fma_peak():
    """(FP64, FP32) FMA throughput of the current GPU in TFLOP/s from the
    separate microbenchmark library (libfma_peak.so), or (None, None)."""
    path = os.path.join(ROOT, "ccpp_physics_b200", "libfma_peak.so")
    try:
        L = ctypes.CDLL(path)
        L.fma_peak_tflops.argtypes = [ctypes.POINTER(ctypes.c_double)] * 2
        p64, p32 = ctypes.c_double(0.0), ctypes.c_double(0.0)
        if L.fma_peak_tflops(ctypes.byref(p64), ctypes.byref(p32)) == 0:
            return p64.value, p32.value
    except OSError:
        pass
    return None, None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch(args):
    """--gpus N > 1 outside a launcher: start N ranks with torch.distributed.run
    (same arguments) and return its exit code."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def dry_run(args, rank, world, local):
    """The multi-rank plumbing alone (no GPU work): process group (NCCL with a
    GPU, gloo without), the max-over-ranks reduction of a per-rank time, and
    rank 0's line with n_gpus."""
    import torch
    import torch.distributed as dist
    use_cuda = torch.cuda.is_available()
    if world > 1:
        if use_cuda:
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if use_cuda else "gloo", timeout=datetime.timedelta(seconds=60))
    dev = torch.device("cuda", local) if use_cuda else torch.device("cpu")
    t = torch.tensor([1.0 + rank], dtype=torch.float64, device=dev)
    seen = torch.tensor([1 << rank], dtype=torch.int64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(seen, op=dist.ReduceOp.SUM)
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        _, mine, c0 = rank_blocks(rank, world)
        print(json.dumps({"dry_run": True, "n_gpus": world, "ranks_seen": int(seen.item()),
                          "max_over_ranks": float(t.item()), "rank0_columns": int(sum(mine)),
                          "config": workload_config(world)}), flush=True)


def run_reference(args, rank, world):
    """Reference arm: the CPU restatement of rrtmg_lw_run (no Fortran compiler
    exists on these machines to build the reference itself) on all host
    threads; each step is one bounded sample of the workload's columns, a
    different one per step."""
    if rank != 0:
        return
    from ccpp_physics_b200 import synthetic
    from oracle import oracle
    ncores = os.cpu_count() or 1
    rc, msg = oracle.rlwinit()
    assert rc == 0, msg
    sample = 16_384
    profs = {}

    def prof(i):
        c0 = (i * sample) % (NCOLS - sample)
        if c0 not in profs:
            profs[c0] = synthetic.make_profiles(sample, NLAY, seed=1, col_offset=c0)
        return profs[c0]
    for i in range(args.warmup):
        oracle.rrtmg_lw_run(synthetic.slice_columns(prof(0), 0, 1024), nthreads=ncores)
    times = []
    for i in range(args.steps):
        p = prof(i)
        t0 = time.perf_counter()
        rc, msg, _ = oracle.rrtmg_lw_run(p, nthreads=ncores)
        times.append(time.perf_counter() - t0)
        assert rc == 0, msg
    rate = sample * len(times) / sum(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "columns/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(world),
        "cpu_baseline": {"value": rate, "unit": "columns/s", "cores": ncores, "kind": "port",
                         "sample": f"{sample} consecutive columns of {WORKLOAD} per step (a different range "
                                   f"each step), OpenMP over columns"},
        "e2e": {"value": rate, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def caller_steps_leg(args, torch, timed, sh, peak_gbs):
    """The steps either side of rrtmg_lw_run at 884,736 columns x 127 layers
    (six C384 cubed-sphere faces of 384 x 384 columns):
      * McICA seeds (GFS_rad_time_vary): one twister stream of 2 x 147,456
        draws per face, then each column's pair; six calls, one per face;
      * decorrelation length (Hogan) + alpha for exponential-random overlap;
      * rrtmg_lw_post_run: heating rates (total and clear sky) onto 127 levels;
      * rrtmg_sw_post_run: the same for the shortwave rates, plus the surface
        component fields, every column daylit;
      * rad_sw_pre_run: the daytime points of all 884,736 columns.
    Device-resident, timed with CUDA events; the oracle times the same work on
    a sample on one host core, and the GPU results are checked against it."""
    import math
    import numpy as np
    from oracle import oracle
    from ccpp_physics_b200 import cloud_overlap, rad_time_vary, rrtmg_lw_post
    n, nlay, cn = 884_736, 127, 384
    face = cn * cn
    k = max(3, min(args.steps, 10))
    g = torch.Generator(device="cuda").manual_seed(11)
    res = {"workload": "c3_884736x127_as_6_c384_faces", "steps": k}

    # seeds: every column of a face, rows of the tile in a shuffled order
    perm = torch.randperm(face, generator=g, device="cuda").to(torch.int32)
    imap, jmap = (perm % cn + 1).contiguous(), (perm // cn + 1).contiguous()
    sw = torch.zeros(face, dtype=torch.int32, device="cuda")
    lwseed = torch.zeros_like(sw)
    sec, ipsd0, ipsdlim = 10800.0, 35000, 100_000_000

    def seeds():
        for _ in range(6):
            m, e = rad_time_vary.gfs_rad_time_vary_seeds(False, None, True, True, 2, 2, sw, lwseed, cn, cn, 1, 1,
                                                         imap, jmap, sec, ipsd0, ipsdlim, stream=sh, sync=False)
            if e:
                raise RuntimeError(m)
    seeds()
    ms = timed(seeds, k)
    t0 = time.perf_counter()
    _, sw_ref, lw_ref = oracle.seeds(sec=sec, ipsd0=ipsd0, ipsdlim=ipsdlim, cnx=cn, cny=cn, isc=1, jsc=1,
                                     imap=imap.cpu().numpy(), jmap=jmap.cpu().numpy())
    cpu_face_s = time.perf_counter() - t0
    res["seeds"] = {"ms_per_step_6_faces": ms / k, "ms_per_face": ms / k / 6, "draws_per_face": 2 * face,
                    "cpu_oracle_ms_per_face": cpu_face_s * 1e3, "cpu_cores": 1,
                    "matches_oracle": bool(np.array_equal(sw.cpu().numpy(), sw_ref)
                                           and np.array_equal(lwseed.cpu().numpy(), lw_ref))}

    # overlap parameters (Hogan length, exponential-random alpha)
    lat = (torch.rand(n, generator=g, device="cuda", dtype=torch.float64) - 0.5) * math.pi
    dz = 0.02 + 2.0 * torch.rand((nlay, n), generator=g, device="cuda", dtype=torch.float64)
    cf = torch.rand((nlay, n), generator=g, device="cuda", dtype=torch.float64)
    cf = torch.where(cf < 0.5, torch.zeros_like(cf), cf)
    dl = torch.zeros(n, dtype=torch.float64, device="cuda")
    al = torch.zeros((nlay, n), dtype=torch.float64, device="cuda")

    def overlap():
        m, e = cloud_overlap.overlap_params(5, 1, dz, cf, dl, al, xlat=lat, stream=sh, sync=False)
        if e:
            raise RuntimeError(m)
    overlap()
    ms = timed(overlap, k)
    ns = 65536
    dz_s, cf_s, lat_s = (dz[:, :ns].cpu().numpy(), cf[:, :ns].cpu().numpy(), lat[:ns].cpu().numpy())
    t0 = time.perf_counter()
    dl_ref, al_ref = oracle.overlap_params(5, 1, dz_s, cf_s, xlat=lat_s)
    cpu_s = time.perf_counter() - t0
    al_g = al[:, :ns].cpu().numpy()
    ulp = np.abs(al_g - al_ref) / np.maximum(np.spacing(np.abs(al_ref)), 5e-324)
    obytes = (3 * nlay + 2) * 8 * n
    res["overlap_params"] = {"ms_per_step": ms / k, "columns_per_s": n * k / (ms / 1e3),
                             "achieved_gbs": obytes * k / (ms / 1e3) / 1e9, "bytes_per_step": obytes,
                             "hbm_frac": obytes * k / (ms / 1e3) / 1e9 / peak_gbs,
                             "cpu_oracle_columns_per_s": ns / cpu_s, "cpu_cores": 1,
                             "cpu_sample": f"first {ns} columns",
                             "de_lgth_matches_oracle": bool(np.array_equal(dl[:ns].cpu().numpy(), dl_ref)),
                             "alpha_max_ulp_vs_oracle": float(ulp.max())}
    del dz, cf, al, lat, dl

    # rrtmg_lw_post_run
    htlwc = torch.randn((nlay, n), generator=g, device="cuda", dtype=torch.float64)
    htlw0 = torch.randn((nlay, n), generator=g, device="cuda", dtype=torch.float64)
    sfc = torch.randn((n, 4), generator=g, device="cuda", dtype=torch.float64)
    tsfa = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    outs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(2)] + \
           [torch.zeros((nlay, n), dtype=torch.float64, device="cuda") for _ in range(2)]

    def post():
        m, e = rrtmg_lw_post.rrtmg_lw_post_run(n, nlay, 0, nlay, 0, True, True, tsfa, htlwc, htlw0, sfc, *outs,
                                               stream=sh, sync=False)
        if e:
            raise RuntimeError(m)
    post()
    ms = timed(post, k)
    sl = [a[..., :ns].cpu().numpy().copy() if a.dim() == 2 else a[:ns].cpu().numpy().copy()
          for a in (htlwc, htlw0)]
    ref = [np.zeros(ns), np.zeros(ns), np.zeros((nlay, ns)), np.zeros((nlay, ns))]
    t0 = time.perf_counter()
    oracle.post(ns, nlay, 0, nlay, 0, 1, 1, tsfa[:ns].cpu().numpy(), sl[0], sl[1], sfc[:ns].cpu().numpy(), *ref)
    cpu_s = time.perf_counter() - t0
    pbytes = (4 * nlay + 3) * 8 * n
    res["post"] = {"ms_per_step": ms / k, "columns_per_s": n * k / (ms / 1e3),
                   "achieved_gbs": pbytes * k / (ms / 1e3) / 1e9, "bytes_per_step": pbytes,
                   "hbm_frac": pbytes * k / (ms / 1e3) / 1e9 / peak_gbs,
                   "cpu_oracle_columns_per_s": ns / cpu_s, "cpu_cores": 1, "cpu_sample": f"first {ns} columns",
                   "matches_oracle": bool(np.array_equal(outs[2][:, :ns].cpu().numpy(), ref[2])
                                          and np.array_equal(outs[3][:, :ns].cpu().numpy(), ref[3]))}
    del htlwc, htlw0, sfc, tsfa, outs

    # rrtmg_sw_post_run, every column daylit (the branch that moves data)
    from oracle import oracle_sw
    from ccpp_physics_b200 import rrtmg_sw_post
    f64 = dict(dtype=torch.float64, device="cuda")
    sins = [torch.rand(n, generator=g, **f64) for _ in range(4)] + \
           [torch.randn((nlay, n), generator=g, **f64) for _ in range(2)]
    souts = [torch.zeros(n, **f64) for _ in range(10)] + [torch.zeros((nlay, n), **f64) for _ in range(2)] + \
            [500 * torch.rand((n, 6), generator=g, **f64), 900 * torch.rand((n, 4), generator=g, **f64),
             torch.zeros((n, 3), **f64)]

    def swpost():
        m, e = rrtmg_sw_post.rrtmg_sw_post_run(n, nlay, nlay, 0, n, nlay, 0, True, True, *sins, *souts,
                                               stream=sh, sync=False)
        if e:
            raise RuntimeError(m)
    swpost()
    ms = timed(swpost, k)
    cut = lambda a: np.ascontiguousarray((a[:, :ns] if a.dim() == 2 and a.shape[0] == nlay else a[:ns]).cpu().numpy())
    sref_in = [cut(a) for a in sins]
    sref_out = [np.zeros_like(cut(a)) for a in souts[:12]] + [cut(a) for a in souts[12:]]
    t0 = time.perf_counter()
    oracle_sw.post(ns, nlay, nlay, 0, ns, nlay, 0, True, True, *sref_in, *sref_out)
    cpu_s = time.perf_counter() - t0
    sbytes = (4 * nlay + 20) * 8 * n    # in: htswc, htsw0, 4 albedos, 4 of scmpsw, 2 of sfcfsw; out: the rest
    res["sw_post"] = {"ms_per_step": ms / k, "columns_per_s": n * k / (ms / 1e3),
                      "achieved_gbs": sbytes * k / (ms / 1e3) / 1e9, "bytes_per_step": sbytes,
                      "hbm_frac": sbytes * k / (ms / 1e3) / 1e9 / peak_gbs,
                      "cpu_oracle_columns_per_s": ns / cpu_s, "cpu_cores": 1, "cpu_sample": f"first {ns} columns",
                      "matches_oracle": bool(all(np.array_equal(cut(a), r) for a, r in zip(souts, sref_out)))}
    del sins, souts

    # rad_sw_pre_run: the daytime points of the whole call (nday read back each call)
    from ccpp_physics_b200 import rad_sw_pre
    cz = 2 * torch.rand(n, generator=g, **f64) - 1
    idx = torch.zeros(n, dtype=torch.int32, device="cuda")
    got = {}

    def swpre():
        nd, m, e = rad_sw_pre.rad_sw_pre_run(n, True, cz, idx, stream=sh)
        if e:
            raise RuntimeError(m)
        got["nday"] = nd
    swpre()
    ms = timed(swpre, k)
    czh = cz.cpu().numpy()
    t0 = time.perf_counter()
    nref, iref = oracle_sw.pre(n, True, czh)
    cpu_s = time.perf_counter() - t0
    pre_bytes = 12 * n                  # coszen in, idxday out
    res["sw_pre"] = {"ms_per_step": ms / k, "columns_per_s": n * k / (ms / 1e3),
                     "achieved_gbs": pre_bytes * k / (ms / 1e3) / 1e9, "bytes_per_step": pre_bytes,
                     "note": "two launches and a 4-byte read-back of nday per call: latency-bound",
                     "cpu_oracle_columns_per_s": n / cpu_s, "cpu_cores": 1, "cpu_sample": f"all {n} columns",
                     "matches_oracle": bool(got["nday"] == nref and np.array_equal(idx.cpu().numpy(), iref))}
    res["peak_gbs"] = peak_gbs
    del cz, idx
    torch.cuda.empty_cache()
    return res


def sw_leg(args, torch, timed, sh):
    """rrtmg_sw_run (radsw_main.F90:493) at 16,384 columns x 127 layers, every
    column daylit, McICA with maximum-random overlap, PIFM two-stream, the
    C2 cloud fields plus aerosols and rain/snow: device-resident inputs timed
    with CUDA events, the host-array call timed end to end, the per-kernel
    split from one call, and the oracle on all host threads as the CPU
    baseline; the GPU fluxes are checked against the oracle's."""
    import ctypes as C
    import numpy as np
    from ccpp_physics_b200 import rrtmg_sw as swm, synthetic
    from oracle import oracle_sw
    n, nlay = args.sw_ncols, 127
    swm.rswinit(device=torch.cuda.current_device())
    prof = swm.add_sw_inputs(synthetic.make_profiles(n, nlay, seed=1), seed=1, precip=True)
    dev = {k: (torch.as_tensor(np.ascontiguousarray(v)).cuda() if isinstance(v, np.ndarray) else v)
           for k, v in prof.items()}
    like = dev["plyr"]
    out = swm.alloc_outputs(n, nlay, like=like)
    keep = []
    a = swm.make_run_args(dev, out, keep=keep)
    x = swm.SwExec(precision=0, memory=1, stream=sh, sync=0)
    buf = C.create_string_buffer(256)

    def step():
        if swm.lib().rrtmg_sw_gpu_run_ex(C.byref(a), C.byref(x), buf, 256):
            raise RuntimeError(buf.value.decode())
    k = max(3, min(args.steps, 10))
    for _ in range(args.warmup):
        step()
    ms = timed(step, k)
    km = (C.c_float * 3)()
    xk = swm.SwExec(precision=0, memory=1, stream=sh, sync=1, kernel_ms=C.cast(km, C.POINTER(C.c_float)))
    if swm.lib().rrtmg_sw_gpu_run_ex(C.byref(a), C.byref(xk), buf, 256):
        raise RuntimeError(buf.value.decode())
    torch.cuda.synchronize()
    got = {kk: v.cpu().numpy() for kk, v in out.items()}
    # the decorrelation-length overlap of GFS v16 (iovr=3, de_lgth 2 km)
    out3 = swm.alloc_outputs(n, nlay, like=like)
    a3 = swm.make_run_args(dev, out3, flags=dict(iovr=3), keep=keep)

    def step3():
        if swm.lib().rrtmg_sw_gpu_run_ex(C.byref(a3), C.byref(x), buf, 256):
            raise RuntimeError(buf.value.decode())
    for _ in range(args.warmup):
        step3()
    ms3 = timed(step3, k)
    km3 = (C.c_float * 3)()
    xk3 = swm.SwExec(precision=0, memory=1, stream=sh, sync=1, kernel_ms=C.cast(km3, C.POINTER(C.c_float)))
    if swm.lib().rrtmg_sw_gpu_run_ex(C.byref(a3), C.byref(xk3), buf, 256):
        raise RuntimeError(buf.value.decode())
    torch.cuda.synchronize()
    got3 = {kk: v.cpu().numpy() for kk, v in out3.items()}
    del out3
    # host arrays (pinned) through the public call, copies in and out inside the timing
    pinned = []

    def pin(v):
        t = torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
        pinned.append(t)
        return t.numpy()
    hprof = {kk: (pin(v) if isinstance(v, np.ndarray) else v) for kk, v in prof.items()}
    hout = {kk: pin(v) for kk, v in swm.alloc_outputs(n, nlay).items()}
    sw_in = ("plyr", "tlyr", "qlyr", "olyr", "gasvmr_co2", "gasvmr_n2o", "gasvmr_ch4", "gasvmr_o2", "aeraod",
             "aerssa", "aerasy", "sfcalb_nir_dir", "sfcalb_nir_dif", "sfcalb_uvis_dir", "sfcalb_uvis_dif", "dzlyr",
             "delpin", "de_lgth", "alpha", "cosz", "cld_cf", "cld_lwp", "cld_ref_liq", "cld_iwp", "cld_ref_ice",
             "cld_rwp", "cld_ref_rain", "cld_swp", "cld_ref_snow", "icseed", "idxday")
    h2d = sum(hprof[kk].nbytes for kk in sw_in)   # the arrays the shortwave call copies in
    d2h = sum(v.nbytes for v in hout.values())
    swm.rrtmg_sw_run(hprof, hout)
    t0 = time.perf_counter()
    for _ in range(3):
        swm.rrtmg_sw_run(hprof, hout)
    e2e_s = (time.perf_counter() - t0) / 3
    e2e_ok = all(np.array_equal(hout[kk], got[kk]) for kk in ("topflx", "sfcflx", "hswc"))
    # CPU baseline + parity: the oracle on every column, all host threads
    oracle_sw.rswinit()
    ref = swm.alloc_outputs(n, nlay)
    t0 = time.perf_counter()
    rc, msg = oracle_sw.run(prof, ref)
    cpu_s = time.perf_counter() - t0
    assert rc == 0, msg
    ref3 = swm.alloc_outputs(n, nlay)
    rc, msg = oracle_sw.run(prof, ref3, flags=dict(iovr=3))
    assert rc == 0, msg
    rel = lambda u, v, f: float(np.max(np.abs(u - v) / np.maximum(np.abs(v), f)))
    # the same columns as uneven physics blocks (8..256 columns, the host's
    # blocking): one rrtmg_sw_gpu_run_blocks call against one call per block
    sizes = synthetic.physics_blocks(n, seed=7)
    bprofs, bouts = [], []
    c0 = 0
    for nb_cols in sizes:
        bp = dict(npts=int(nb_cols), nlay=nlay, solcon=prof["solcon"], sw_flags=prof["sw_flags"])
        for kk, v in prof.items():
            if isinstance(v, np.ndarray) and v.shape[-1] == n:
                bp[kk] = torch.as_tensor(np.ascontiguousarray(v[..., c0:c0 + nb_cols])).cuda()
        idx = prof["idxday"]
        bp["idxday"] = torch.as_tensor((idx[(idx > c0) & (idx <= c0 + nb_cols)] - c0).astype(np.int32)).cuda()
        bprofs.append(bp)
        bouts.append(swm.alloc_outputs(int(nb_cols), nlay, like=like))
        c0 += nb_cols
    arr = (swm.SwRunArgs * len(sizes))()
    for b in range(len(sizes)):
        arr[b] = swm.make_run_args(bprofs[b], bouts[b], keep=keep)

    def step_blocks():
        if swm.lib().rrtmg_sw_gpu_run_blocks(arr, len(sizes), C.byref(x), buf, 256):
            raise RuntimeError(buf.value.decode())

    def step_per_block():
        for b in range(len(sizes)):
            if swm.lib().rrtmg_sw_gpu_run_ex(C.byref(arr[b]), C.byref(x), buf, 256):
                raise RuntimeError(buf.value.decode())
    for _ in range(args.warmup):
        step_blocks()
    ms_bl = timed(step_blocks, k)
    step_per_block()
    kp = max(2, k // 2)
    ms_pb = timed(step_per_block, kp)
    blocks_ok = all(np.array_equal(bouts[b]["topflx"].cpu().numpy(), got["topflx"][int(sum(sizes[:b])):int(sum(sizes[:b + 1]))])
                    for b in range(len(sizes)))
    del bprofs, bouts
    # roofline of the dominant (transfer) kernel: counted flops and DRAM bytes per
    # column from the ncu capture, against the FMA peak measured now and the
    # measured copy bandwidth
    roof = None
    try:
        tf = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "sw_kernels_traffic.txt")
        with open(tf) as fh:
            tr = {kk.strip(): float(v) for kk, v in (l.split(":", 1) for l in fh if ":" in l and not l.startswith("#"))}
        p64v, _ = fma_peak()
        rc_peak = 0 if p64v else 1
        p64 = C.c_double(p64v or 0.0)
        t_rt = km[2] / 1e3
        ach_tf = tr["sw_fp64_flop_per_column_rt"] * n / t_rt / 1e12
        ach_gbs = tr["sw_dram_bytes_per_column_rt"] * n / t_rt / 1e9
        hbm = _peaks()[0]
        roof = {"kernel": "sw_rt_kernel<false>", "fp64_tflops": ach_tf,
                "fp64_peak_tflops": p64.value if rc_peak == 0 else None,
                "fp64_frac": ach_tf / p64.value if rc_peak == 0 and p64.value > 0 else None,
                "dram_gbs": ach_gbs, "hbm_peak_gbs": hbm, "hbm_frac": ach_gbs / hbm if hbm else None,
                "source": "per-column flops and DRAM bytes: profiles/sw_kernels_traffic.txt (ncu); kernel time: "
                          "CUDA events of this run; FP64 peak: FMA-chain kernel in this run"}
    except Exception as exc:   # report, never fake
        roof = {"unavailable": str(exc)}
    return {"workload": f"sw_c2_allsky_mcica_{n}x127", "steps": k, "roofline": roof, "value": n * k / (ms / 1e3),
            "unit": "columns/s", "ms_per_step": ms / k,
            "kernel_ms": {"optics": km[1], "mcica": km[0], "transfer": km[2]},
            "blocks": {"nblocks": len(sizes), "block_sizes": "8..256 (physics_blocks seed 7)",
                       "run_blocks_columns_per_s": n * k / (ms_bl / 1e3),
                       "per_block_calls_columns_per_s": n * kp / (ms_pb / 1e3),
                       "matches_single_call": bool(blocks_ok)},
            "e2e_columns_per_s": n / e2e_s, "e2e_h2d_bytes": h2d, "e2e_d2h_bytes": d2h,
            "e2e_matches_device_run": e2e_ok,
            "flux_max_rel_vs_oracle": max(rel(got[kk], ref[kk], 1e-300) for kk in ("topflx", "sfcflx", "fdncmp")),
            "hr_max_rel_vs_oracle": max(rel(got[kk], ref[kk], 1.0) for kk in ("hswc", "hsw0")),
            "iovr3": {"value": n * k / (ms3 / 1e3), "ms_per_step": ms3 / k,
                      "kernel_ms": {"optics": km3[1], "mcica": km3[0], "transfer": km3[2]},
                      "flux_max_rel_vs_oracle": max(rel(got3[kk], ref3[kk], 1e-300) for kk in ("topflx", "sfcflx")),
                      "overlap": "decorrelation length (iovr=3), de_lgth 2 km"},
            "cpu_oracle_columns_per_s": n / cpu_s, "cpu_cores": os.cpu_count(),
            "cpu_sample": f"all {n} columns, OpenMP over columns",
            "flags": "iovr=1 isubcsw=2 iswcliq=1 iswcice=3 iswmode=2, aerosols, rain+snow, all columns daylit"}


def training_leg(args, torch, sg):
    """Learned gas optics training throughput on 20M layer samples labelled by
    plain FP64 taumol: a fresh network, 2 epochs of the library's tcgen05
    forward/backward kernels + Adam (batch 8,192).  The committed network
    (trained the same way for 100 epochs) is reloaded afterwards."""
    t0 = time.time()
    feats, targ = sg.make_dataset(20_000_000, seed=101)
    norm = sg.normalisation(feats, targ)
    y = sg.normalise_targets(targ, norm)
    del targ
    torch.cuda.synchronize()
    t_data = time.time() - t0
    sg.init(norm, seed=1)
    epochs = 2
    t0 = time.time()
    losses = sg.train(feats, y, epochs=epochs, batch=8192, lr=3e-3, lr_final=1e-5, tau_weight=True)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    n = feats.shape[0]
    del feats, y
    torch.cuda.empty_cache()
    meta = sg.load()
    flop = 2 * (16 * 128 + 128 * 128 + 128 * 288) + 2 * (2 * 288 * 128 + 2 * 128 * 128 + 128 * 16)   # padded fwd + bwd
    return {"workload": "c4_surrogate_training_20M", "samples": int(n), "epochs": epochs, "batch": 8192,
            "data_s": round(t_data, 2), "train_s": round(t_train, 2),
            "samples_per_s": n * epochs / t_train, "tflops": n * epochs * flop / t_train / 1e12,
            "loss_first_epoch": float(losses[0]), "loss_last_epoch": float(losses[-1]),
            "shipped_network": {"epochs": int(meta["epochs"]), "train_s": float(meta["train_seconds"]),
                                "final_loss": float(meta["losses"][-1])}}


def _rel(a, b, floor):
    import numpy as np
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


def parity_check(gpu, ref, ncheck, c_start, flux_keys=("topflx", "sfcflx"), tol=1e-10):
    """Max relative difference of the GPU FP64 outputs (numpy, first ncheck
    columns) from the oracle's; the columns over `tol` are counted and the
    first few named by global index."""
    import numpy as np
    bad = np.zeros(ncheck, dtype=bool)
    fmax = 0.0
    for k in flux_keys:
        r = _rel(gpu[k], ref[k], 1e-300)
        fmax = max(fmax, float(r.max()))
        col_axis = 1 if k == "flxprf" else 0
        rr = r.reshape(r.shape[0], -1) if col_axis == 0 else np.moveaxis(r, 1, 0).reshape(ncheck, -1)
        bad |= rr.max(axis=1) > tol
    hmax = 0.0
    for k in ("hlwc", "hlw0"):
        r = _rel(gpu[k], ref[k], 1.0)   # K/day, floored at 1 K/day as in the parity tests
        hmax = max(hmax, float(r.max()))
    idx = np.nonzero(bad)[0]
    return {"flux_max_rel": fmax, "hr_max_rel": hmax, "cols": ncheck, "cols_over_1e-10": int(idx.size),
            "cols_over_named": [int(c_start + i) for i in idx[:8]]}


def headline(args, rank, world, local, dist, torch, sh, stream, lw, abi, synthetic):
    """The default workload on this rank's blocks: FP64 (the headline value),
    FP32 and the learned gas optics, parity against the oracle, end to end
    from pinned host memory, roofline and CPU baseline."""
    import ctypes as C
    import numpy as np

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def maxr(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(fn, k):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        barrier()
        return maxr(e0.elapsed_time(e1))

    def rmse(a, b):
        return float(torch.sqrt(torch.mean((a - b) ** 2)).item())

    _, sizes, c_start = rank_blocks(rank, world)
    ncols = int(np.sum(sizes))
    prof = synthetic.make_profiles(ncols, NLAY, seed=1, cloudy=True, col_offset=c_start, device="cuda")
    # pinned host copy (the caller's Fortran arrays) for the end-to-end leg
    hprof, h2d = None, 0
    if not args.no_e2e:
        hprof = dict(npts=ncols, nlay=NLAY, flags=dict(prof["flags"]))
        for k, v in prof.items():
            if isinstance(v, torch.Tensor):
                hv = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                hv.copy_(v)
                hprof[k] = hv
                h2d += hv.numel() * hv.element_size()
    lw.pack_blocks(prof, sizes, inplace=True)
    torch.cuda.empty_cache()

    k_main = args.steps
    k_other = max(3, min(args.steps, 10))
    res, outs = {}, {}
    from ccpp_physics_b200 import surrogate as sg
    try:
        sg.load()
        precs = ("fp64", "fp32", "surrogate")
    except Exception as exc:   # weights missing: report, do not fake
        res["surrogate"] = {"value": None, "note": f"no trained network: {exc}"}
        precs = ("fp64", "fp32")
    clk = None
    buf = C.create_string_buffer(512)
    for prec in precs:
        out = lw.pack_blocks(abi.alloc_outputs(ncols, NLAY, hlw0=True, like="cuda"), sizes, inplace=True)
        best, _ = lw.autotune(prof, out, sizes, precision=prec, sample_cols=65536, stream=sh)
        arr, keep = lw.block_args(prof, out, sizes)
        x = abi.ExecArgs(precision=lw.PRECISIONS[prec], memory=abi.DEVICE, stream=sh, sync=0)
        tun = abi.Tuning(**dict(best, use_graph=1))

        def call():
            if lw.lib().rrtmg_lw_gpu_run_blocks(arr, len(arr), C.byref(x), C.byref(tun), buf, 512):
                raise RuntimeError(buf.value.decode())
        for _ in range(args.warmup):
            call()
        if prec == "surrogate":
            sg.stats(reset=True)
        if prec == "fp64":
            with ClockSampler(local) as clk:
                ms = timed(call, k_main)
            k = k_main
        else:
            ms = timed(call, k_other)
            k = k_other
        launches = int(lw.lib().rrtmg_lw_gpu_last_launch_count())
        # per-kernel device times of one call without the graph
        kms = (C.c_float * 3)()
        xk = abi.ExecArgs(precision=lw.PRECISIONS[prec], memory=abi.DEVICE, stream=sh, sync=1,
                          kernel_ms=C.cast(kms, C.POINTER(C.c_float)))
        tk = abi.Tuning(**dict(best, use_graph=0))
        if lw.lib().rrtmg_lw_gpu_run_blocks(arr, len(arr), C.byref(xk), C.byref(tk), buf, 512):
            raise RuntimeError(buf.value.decode())
        r = {"value": NCOLS * k / (ms / 1e3), "ms_per_step": ms / k, "steps": k, "launches_per_step": launches,
             "mcica_ms": kms[0], "tuning": {kk: int(v) for kk, v in best.items()}}
        if prec == "surrogate":
            fb, mma_err = sg.stats()
            r["fallback_layer_frac"] = fb / float(k * ncols * NLAY)
            r["mma_error"] = mma_err
        res[prec] = r
        outs[prec] = out
    b = outs["fp64"]
    for prec in precs[1:]:
        a = outs[prec]
        res[prec].update({
            "speedup_vs_fp64": res[prec]["value"] / res["fp64"]["value"],
            "flux_rmse_wm2": rmse(torch.cat([a["topflx"], a["sfcflx"]], 1), torch.cat([b["topflx"], b["sfcflx"]], 1)),
            "hr_rmse_kday": rmse(a["hlwc"], b["hlwc"]), "hr0_rmse_kday": rmse(a["hlw0"], b["hlw0"])})
        del a
        outs[prec] = None
    # FP64 outputs in the caller's (unpacked) layout, on the host
    gpu64 = {kk: v.cpu().numpy() for kk, v in lw.unpack_blocks(outs["fp64"]).items()}
    del outs, b, prof
    torch.cuda.empty_cache()

    # ---- end to end: rrtmg_lw_gpu_run on pinned host arrays ----
    e2e = None
    if hprof is not None:
        hout = {kk: torch.empty(v.shape, dtype=torch.float64, pin_memory=True) for kk, v in gpu64.items()}
        d2h = sum(v.numel() * v.element_size() for v in hout.values())
        m, e = lw.run_profile(hprof, hout, precision="fp64")
        assert e == 0, m
        ke = max(1, min(args.steps, 3))
        barrier()
        t0 = time.perf_counter()
        for _ in range(ke):
            m, e = lw.run_profile(hprof, hout, precision="fp64")
            assert e == 0, m
        t_e2e = maxr(time.perf_counter() - t0)
        e2e = {"value": NCOLS * ke / t_e2e, "unit": "columns/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": ke,
               "matches_device_run": bool(all(np.array_equal(hout[kk].numpy(), gpu64[kk]) for kk in hout))}
        del hprof, hout

    # ---- parity against the oracle + CPU baseline (rank 0) ----
    parity, cpu = None, None
    if rank == 0 and not args.no_parity:
        from oracle import oracle
        rc, msg = oracle.rlwinit()
        assert rc == 0, msg
        ncores = os.cpu_count() or 1
        ns = min(ncols, PARITY_SAMPLE)
        pnp = synthetic.make_profiles(ns, NLAY, seed=1, col_offset=c_start)
        t0 = time.perf_counter()
        rc, msg, ref = oracle.rrtmg_lw_run(pnp, hlw0=True, flxprf=True, nthreads=ncores)
        dt = time.perf_counter() - t0
        assert rc == 0, msg
        cpu = {"value": ns / dt, "unit": "columns/s", "cores": ncores, "kind": "port",
               "sample": f"first {ns} columns of {WORKLOAD} ({dt:.1f} s), OpenMP over columns"}
        sub = {kk: (v[:ns] if kk in ("topflx", "sfcflx") else v[:, :ns]) for kk, v in gpu64.items()}
        parity = {"c3_first_%d" % ns: parity_check(sub, ref, ns, c_start)}
        # the 16,384-column all-sky case as one call, flux profiles included
        n2 = min(ns, C2_COLS)
        p2 = synthetic.make_profiles(n2, NLAY, seed=1, col_offset=c_start, device="cuda")
        o2 = abi.alloc_outputs(n2, NLAY, hlw0=True, flxprf=True, like="cuda")
        m, e = lw.run_profile(p2, o2, precision="fp64")
        assert e == 0, m
        g2 = {kk: v.cpu().numpy() for kk, v in o2.items()}
        r2 = {kk: (v[:n2] if kk in ("topflx", "sfcflx") else v[:, :n2] if kk != "flxprf" else v[:, :n2, :])
              for kk, v in ref.items()}
        parity["c2_%d" % n2] = parity_check(g2, r2, n2, c_start, flux_keys=("topflx", "sfcflx", "flxprf"))
        del p2, o2
    return res, e2e, parity, cpu, clk, ncols


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--legs", default="", help="comma list of auxiliary legs printed before the headline: "
                                                "sw, callers, train")
    ap.add_argument("--only-legs", action="store_true", help="print the --legs lines and stop (no headline); "
                                                              "profiling runs of the auxiliary legs")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end host-memory leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the oracle parity check and CPU baseline")
    ap.add_argument("--dry-run", action="store_true", help="launcher and process-group plumbing only")
    ap.add_argument("--ncols", type=int, default=0, help="profiling runs: one device-resident call of the "
                                                         "first NCOLS columns, --precision, no other legs")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32", "surrogate"])
    ap.add_argument("--sw-ncols", type=int, default=16384, help="columns of the shortwave leg")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.dry_run:
        dry_run(args, rank, world, local)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    from ccpp_physics_b200 import abi, synthetic
    from ccpp_physics_b200 import rrtmg_lw as lw

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    rc, msg = lw.rlwinit(device=local, me=1)   # me != 0: no banner, stdout carries only JSON lines
    assert rc == 0, msg
    # a dedicated stream: the library and the CUDA events must share it (the
    # legacy default stream does not order work of non-blocking streams)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    def timed(fn, k):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    if args.ncols:
        # profiling runs: one path over the first NCOLS columns, device resident
        import ctypes as C
        prof = synthetic.make_profiles(args.ncols, NLAY, seed=1, device="cuda")
        out = abi.alloc_outputs(args.ncols, NLAY, hlw0=True, like="cuda")
        if args.precision == "surrogate":
            from ccpp_physics_b200 import surrogate as sg
            sg.load()
        keep = []
        a = abi.make_run_args(prof, out, keep=keep)
        x = abi.ExecArgs(precision=lw.PRECISIONS[args.precision], memory=abi.DEVICE, stream=sh, sync=0)
        buf = C.create_string_buffer(512)

        def step():
            if lw.lib().rrtmg_lw_gpu_run_ex(C.byref(a), C.byref(x), buf, 512):
                raise RuntimeError(buf.value.decode())
        for _ in range(args.warmup):
            step()
        ms = timed(step, args.steps)
        if rank == 0:
            print(json.dumps({"profiling_run": True, "precision": args.precision, "ncols": args.ncols,
                              "value": world * args.ncols * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                              "launches_per_step": int(lw.lib().rrtmg_lw_gpu_last_launch_count())}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    legs = [l for l in args.legs.split(",") if l]
    if legs and world == 1 and rank == 0:
        peak_gbs = _peaks()[0]
        if "sw" in legs:
            print(json.dumps({"leg": "rrtmg_sw", **sw_leg(args, torch, timed, sh)}), flush=True)
        if "callers" in legs:
            print(json.dumps({"leg": "caller_steps", **caller_steps_leg(args, torch, timed, sh, peak_gbs)}),
                  flush=True)
        if "train" in legs:
            from ccpp_physics_b200 import surrogate as sg
            print(json.dumps({"leg": "c4_training", **training_leg(args, torch, sg)}), flush=True)
        torch.cuda.empty_cache()
    if args.only_legs:
        if dist is not None:
            dist.destroy_process_group()
        return

    res, e2e, parity, cpu, clk, ncols = headline(args, rank, world, local, dist, torch, sh, stream, lw, abi,
                                                 synthetic)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peak, peak_kind = _peaks()
    r64 = res["fp64"]
    # the column kernels (gas optics + transfer, every chunk) take the step
    # minus the McICA kernel; their algorithmic bytes are the interface bytes
    col_s = max(1e-9, (r64["ms_per_step"] - r64["mcica_ms"]) / 1e3)
    achieved = BYTES_PER_COL * ncols / col_s / 1e9
    traffic, fp_pipe, tr = None, None, {}
    tfile = os.path.join(ROOT, "profiles", "column_kernels_traffic.txt")
    if os.path.exists(tfile):
        with open(tfile) as fh:
            tr = dict(l.split(":", 1) for l in fh if ":" in l and not l.startswith("#"))
        if "dram_bytes_per_column_fp64" in tr:
            nch = max(1, (r64["launches_per_step"] - 1) // 2)
            traffic = float(tr["dram_bytes_per_column_fp64"]) * ncols / nch   # per launch pair
    try:
        flop_col = sum(float(tr[k]) for k in ("fp64_flop_per_column_mcica", "fp64_flop_per_column_gas",
                                              "fp64_flop_per_column_rt"))
        p64, p32 = fma_peak()
        if p64:
            ach = flop_col * ncols / (r64["ms_per_step"] / 1e3) / 1e12
            fp_pipe = {"achieved_tflops": ach, "peak_tflops": p64, "frac": ach / p64,
                       "flop_per_column": flop_col}
    except Exception as exc:   # report, never fake
        fp_pipe = {"unavailable": str(exc)[:80]}
    paths = {"fp64": {"value": r64["value"], "ms_per_step": r64["ms_per_step"], "launches": r64["launches_per_step"],
                      "mcica_ms": r64["mcica_ms"]}}
    for prec in ("fp32", "surrogate"):
        if prec in res and res[prec].get("value"):
            p = res[prec]
            paths[prec] = {kk: p[kk] for kk in ("value", "ms_per_step", "speedup_vs_fp64", "flux_rmse_wm2",
                                                "hr_rmse_kday", "hr0_rmse_kday", "launches_per_step")}
            if prec == "surrogate":
                paths[prec]["fallback_layer_frac"] = p["fallback_layer_frac"]
                paths[prec]["mma_error"] = p["mma_error"]
        elif prec in res:
            paths[prec] = res[prec]
    rec = {
        "metric": METRIC, "value": r64["value"], "unit": "columns/s", "n_gpus": world, "steps": r64["steps"],
        "warmup": args.warmup, "ms_per_step": r64["ms_per_step"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(world),
        "gpu_launches": r64["steps"] * r64["launches_per_step"],
        "clocks": clk.summary() if clk else None,
        "e2e": e2e,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "kernel": "lw_gas_kernel<double,4> + lw_rt_kernel<double,4> (per chunk)"},
        "fp_pipe": fp_pipe,
        "cpu_baseline": cpu,
        "paths": paths,
        "parity_fp64_vs_oracle": parity,
    }
    print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    main()
