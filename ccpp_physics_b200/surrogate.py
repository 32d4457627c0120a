"""Learned gas optics for the RRTMG-LW path (host side).

The network (8 -> 128 -> 128 -> 288, SiLU, BF16 tensor-core kernels in
csrc/lw_mlp.cu) maps the intensive state of a layer to the 140 g-point
log(taug/coldry) and the 140 Planck fractions that setcoef + taumol
(radlw_main.F90:2151-2406, 3836-6840) compute.  Training data come from the
library's own plain taumol on the GPU (rrtmg_lw_gpu_gas_optics), features
from rrtmg_lw_gpu_surrogate_features; training runs in the library
(rrtmg_lw_gpu_surrogate_train: hand-written forward, backward and Adam
kernels).  Layers whose features leave the training envelope fall back to
plain taumol inside the column path.

Everything here is plumbing around those entry points: it allocates device
tensors, computes normalisation statistics and moves weights in and out.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi, synthetic

NORM = 608
NPARAM = 53656
NGRAD = 54688
NSTATE = 54688   # parameters and each Adam moment, padded layout (rrtmg_lw_gpu_surrogate_get_state)
NOUTP = 288
NGPT = 140
TAU = slice(0, 140)
FRAC = slice(144, 284)
# Floor of the log(taug/coldry) targets: below it a layer's optical depth
# (coldry is ~200 per hPa of layer thickness) is < 1e-8 and irrelevant, while
# exact zeros (bands without an absorber above laytrop) would otherwise sit
# at log(tiny) and dominate the output scaling of their g-points.
LOG_TAU_FLOOR = -25.0

WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "lw_surrogate_weights.npz")


def _lib():
    from . import rrtmg_lw as lw
    L = lw.lib()
    if not getattr(L, "_sg_bound", False):
        L.rrtmg_lw_gpu_surrogate_features.argtypes = [C.POINTER(abi.RunArgs), C.c_void_p, C.c_void_p, C.c_void_p,
                                                      C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_init.argtypes = [C.c_void_p, C.c_uint64, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_set.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_get.argtypes = [C.c_void_p, C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_train.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32,
                                                   C.c_float, C.c_float, C.c_uint64, C.c_int32, C.c_void_p,
                                                   C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_forward.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_char_p,
                                                     C.c_int32]
        L.rrtmg_lw_gpu_surrogate_grads.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                                   C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_stats.argtypes = [C.POINTER(C.c_uint64), C.POINTER(C.c_int32), C.c_int32]
        L.rrtmg_lw_gpu_surrogate_get_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_int64),
                                                       C.c_void_p, C.c_char_p, C.c_int32]
        L.rrtmg_lw_gpu_surrogate_set_state.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                                       C.c_char_p, C.c_int32]
        L._sg_bound = True
    return L


def _check(rc, msg):
    if rc:
        from .rrtmg_lw import RRTMGLWError
        raise RRTMGLWError(msg.value.decode())


def _stream(stream, x):
    from .rrtmg_lw import torch_stream
    return torch_stream(stream, x)


def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def features(prof: dict, stream=None):
    """(feats [npts*nlay, 8], coldry [npts*nlay]) float32 CUDA tensors of a
    device-resident profile dict; rows are column-major over (column, layer),
    layers surface first."""
    import torch
    n = prof["npts"] * prof["nlay"]
    dev = prof["plyr"].device
    feats = torch.empty((n, 8), dtype=torch.float32, device=dev)
    coldry = torch.empty((n,), dtype=torch.float32, device=dev)
    keep = []
    a = abi.make_run_args(prof, {}, keep=keep)
    stream = _stream(stream, prof["plyr"])
    msg = C.create_string_buffer(512)
    rc = _lib().rrtmg_lw_gpu_surrogate_features(C.byref(a), C.c_void_p(feats.data_ptr()),
                                                C.c_void_p(coldry.data_ptr()), stream, msg, 512)
    _check(rc, msg)
    return feats, coldry


def targets_of(taug, fracs, coldry):
    """Raw (unnormalised) padded targets [n, 288] from plain-taumol outputs
    taug/fracs [npts, nlay, 140] and coldry [npts*nlay]."""
    import torch
    n = coldry.numel()
    t = torch.zeros((n, NOUTP), dtype=torch.float32, device=coldry.device)
    tg = taug.reshape(n, NGPT)
    t[:, TAU] = torch.clamp(torch.log(torch.clamp(tg / coldry.double()[:, None], min=1e-300)),
                            min=LOG_TAU_FLOOR).float()
    t[:, FRAC] = fracs.reshape(n, NGPT).float()
    return t


def make_dataset(nsamples: int, *, seed: int = 101, nlay: int = 127, chunk_cols: int = 8192, device="cuda"):
    """Training set from the synthetic profile generator (clear and cloudy
    columns alike: gas optics does not see clouds).  Returns feats [n, 8]
    (slot 7 holds the layer's coldry) and raw targets [n, 288] (float32 CUDA
    tensors), n = whole columns covering nsamples layers."""
    import torch
    from . import rrtmg_lw as lw
    ncols = -(-nsamples // nlay)
    feats = torch.empty((ncols * nlay, 8), dtype=torch.float32, device=device)
    targ = torch.empty((ncols * nlay, NOUTP), dtype=torch.float32, device=device)
    for c0 in range(0, ncols, chunk_cols):
        nc = min(chunk_cols, ncols - c0)
        prof = synthetic.make_profiles(nc, nlay, seed=seed, col_offset=c0, cloudy=False, device=device)
        f, cd = features(prof)
        taug, fracs = lw.gas_optics(prof, precision="fp64")
        r0, r1 = c0 * nlay, (c0 + nc) * nlay
        f[:, 7] = cd          # the network ignores slot 7 (its bias input is a constant 1); training weights use it
        feats[r0:r1] = f
        targ[r0:r1] = targets_of(taug, fracs, cd)
        del prof, taug, fracs
    return feats, targ


def normalisation(feats, targ, *, margin=0.0):
    """float32[608]: input mean/std, envelope low/high (feature min/max over
    the training set, widened by `margin` of the range) and output mean/std."""
    import torch
    norm = np.zeros(NORM, dtype=np.float32)
    f = feats[:, :7].double()
    mu, sd = f.mean(0), f.std(0)
    lo, hi = f.min(0).values, f.max(0).values
    rng = hi - lo
    sd = torch.where(sd > 1e-6 * torch.clamp(mu.abs(), min=1.0), sd, torch.ones_like(sd))
    norm[0:7] = mu.cpu().numpy()
    norm[8:15] = sd.cpu().numpy()
    norm[7], norm[15] = 0.0, 1.0
    norm[16:23] = (lo - margin * rng).cpu().numpy()
    norm[24:31] = (hi + margin * rng).cpu().numpy()
    norm[23], norm[31] = 1.0, 1.0
    t = targ.double()
    om, osd = t.mean(0), t.std(0)
    osd = torch.where(osd > 1e-6, osd, torch.ones_like(osd))
    norm[32:32 + NOUTP] = om.cpu().numpy()
    norm[32 + NOUTP:] = osd.cpu().numpy()
    pad = np.r_[140:144, 284:288]
    norm[32 + pad] = 0.0
    norm[32 + NOUTP + pad] = 1.0
    return norm


def normalise_targets(targ, norm):
    """Targets in the network's output space (z-scores; padding 0)."""
    import torch
    mu = torch.from_numpy(norm[32:32 + NOUTP]).to(targ.device)
    sd = torch.from_numpy(norm[32 + NOUTP:]).to(targ.device)
    y = (targ - mu) / sd
    y[:, 140:144] = 0
    y[:, 284:] = 0
    return y.contiguous()


def init(norm, seed=1):
    msg = C.create_string_buffer(512)
    n = np.ascontiguousarray(norm, dtype=np.float32)
    _check(_lib().rrtmg_lw_gpu_surrogate_init(_np_ptr(n), seed, msg, 512), msg)


def set_weights(w, norm):
    msg = C.create_string_buffer(512)
    w = np.ascontiguousarray(w, dtype=np.float32)
    n = np.ascontiguousarray(norm, dtype=np.float32)
    assert w.size == NPARAM and n.size == NORM
    _check(_lib().rrtmg_lw_gpu_surrogate_set(_np_ptr(w), _np_ptr(n), msg, 512), msg)


def get_weights():
    w = np.zeros(NPARAM, dtype=np.float32)
    n = np.zeros(NORM, dtype=np.float32)
    msg = C.create_string_buffer(512)
    _check(_lib().rrtmg_lw_gpu_surrogate_get(_np_ptr(w), _np_ptr(n), msg, 512), msg)
    return w, n


def train(feats, ytarg, *, epochs=4, batch=8192, lr=2e-3, lr_final=1e-5, seed=7, tau_weight=False, stream=None):
    """Adam training in the library; returns the per-epoch (weighted) MSE.
    tau_weight: weight optical-depth errors by 1/(1+1.66 tau); needs the
    layer coldry in feats[:, 7] (make_dataset stores it there)."""
    losses = np.zeros(epochs, dtype=np.float32)
    stream = _stream(stream, feats)
    msg = C.create_string_buffer(512)
    rc = _lib().rrtmg_lw_gpu_surrogate_train(C.c_void_p(feats.data_ptr()), C.c_void_p(ytarg.data_ptr()),
                                             feats.shape[0], epochs, batch, lr, lr_final, seed, int(bool(tau_weight)),
                                             _np_ptr(losses),
                                             stream, msg, 512)
    _check(rc, msg)
    return losses


def forward(feats, stream=None):
    import torch
    y = torch.empty((feats.shape[0], NOUTP), dtype=torch.float32, device=feats.device)
    stream = _stream(stream, feats)
    msg = C.create_string_buffer(512)
    rc = _lib().rrtmg_lw_gpu_surrogate_forward(C.c_void_p(feats.data_ptr()), feats.shape[0],
                                               C.c_void_p(y.data_ptr()), stream, msg, 512)
    _check(rc, msg)
    return y


def grads(feats, ytarg, batch):
    g = np.zeros(NGRAD, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    msg = C.create_string_buffer(512)
    rc = _lib().rrtmg_lw_gpu_surrogate_grads(C.c_void_p(feats.data_ptr()), C.c_void_p(ytarg.data_ptr()), batch,
                                             _np_ptr(g), _np_ptr(loss), _stream(None, feats), msg, 512)
    _check(rc, msg)
    return g, float(loss[0])


def stats(reset=False):
    """(layers that fell back to taumol since the last reset, MMA error flag)."""
    n = C.c_uint64(0)
    e = C.c_int32(0)
    if _lib().rrtmg_lw_gpu_surrogate_stats(C.byref(n), C.byref(e), int(reset)):
        raise RuntimeError("surrogate stats unavailable")
    return int(n.value), int(e.value)


def get_state():
    """Training state: dict(params, m, v: float32[NSTATE], step, norm)."""
    st = {k: np.zeros(NSTATE, dtype=np.float32) for k in ("params", "m", "v")}
    norm = np.zeros(NORM, dtype=np.float32)
    step = C.c_int64(0)
    msg = C.create_string_buffer(512)
    _check(_lib().rrtmg_lw_gpu_surrogate_get_state(_np_ptr(st["params"]), _np_ptr(st["m"]), _np_ptr(st["v"]),
                                                   C.byref(step), _np_ptr(norm), msg, 512), msg)
    st.update(step=int(step.value), norm=norm)
    return st


def set_state(params, m, v, step, norm):
    """Restore a training state (get_state's fields): training resumes
    with the same parameters, Adam moments and step count."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (params, m, v)]
    n = np.ascontiguousarray(norm, dtype=np.float32)
    if any(a.size != NSTATE for a in arrs) or n.size != NORM:
        raise ValueError(f"training state arrays must hold {NSTATE} values (norm {NORM})")
    msg = C.create_string_buffer(512)
    _check(_lib().rrtmg_lw_gpu_surrogate_set_state(_np_ptr(arrs[0]), _np_ptr(arrs[1]), _np_ptr(arrs[2]),
                                                   int(step), _np_ptr(n), msg, 512), msg)


def save_checkpoint(path, **meta):
    """Training checkpoint (.npz): parameters, Adam moments, step,
    normalisation and any extra metadata."""
    st = get_state()
    np.savez_compressed(path, params=st["params"], m=st["m"], v=st["v"], step=np.int64(st["step"]),
                        norm=st["norm"], **meta)


def load_checkpoint(path):
    """Restore a checkpoint written by save_checkpoint; returns its contents."""
    d = np.load(path)
    set_state(d["params"], d["m"], d["v"], int(d["step"]), d["norm"])
    return d


def save(path=WEIGHTS_PATH, **meta):
    w, n = get_weights()
    np.savez_compressed(path, weights=w, norm=n, **meta)


def load(path=WEIGHTS_PATH):
    d = np.load(path)
    set_weights(d["weights"], d["norm"])
    return d
