"""Learned warm start: a 3-D convolutional encoder-decoder that predicts the coarsest scale level's
kernel weights alpha from an image pair (no counterpart in the reference).

The plain method (src/SKMReg.cxx:123-470) starts every level from alpha = 0.  Here a small network
maps the (fixed, moving) pair to the alpha grid of the first level, and the scale loop starts that
level from it (skm_register's first_level_parameters); the plain optimizer still runs every later
level, stays the fallback (zeros) when the prediction does not lower the first level's metric value,
and its final metric value is what a warm-started run is judged by.

Network (channels-last bf16 activations, FP32 accumulation, every convolution 3x3x3 padding 1):
    encoder  2 -> 16 -> 32 -> 64 -> 128 channels, stride 2 each (96x96x64 -> 6x6x4)
    decoder  128 -> 64 (stride 1) -> 3 (stride 1, linear): the alpha grid of the first level
             (control spacing 16 voxels at 96x96x64: 6x6x4 points, 3 components)
Every convolution runs on the project's tcgen05 kernels (include/skm_warmstart.h,
csrc/skm_conv.cu): forward, data gradient and weight gradient; Adam and the MSE loss are CUDA
kernels of the same library.  torch only holds device memory and streams.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from . import abi
from .evaluator import check, lib

LAYERS = [(2, 16, 2, True), (16, 32, 2, True), (32, 64, 2, True), (64, 128, 2, True), (128, 64, 1, True),
          (64, 3, 1, False)]
INPUT_SIZE = (96, 96, 64)          # x, y, z voxels
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "warmstart_weights.npz")

# the first scale level whose alpha the network predicts: level 0 of the bench's multi-scale
# configuration (sigma_C4 48, sigma_C0 96, control spacing 48 / 3 = 16 voxels)
LEVEL0 = dict(num_scales=1, sigma_C4=[48], sigma_C0=[96], cp_spacing_scaler=3.0, smoothing_variance=[2],
              sampling_rate=[1], neighborhood_sampling=[1], num_function_evaluations=[100], metric="ncc",
              reg_rd=[1e-3], initial_step_size=[1000.0], tensor_weights=[0])
MS_CONFIG = dict(num_scales=3, sigma_C4=[48, 24, 12], sigma_C0=[96, 48, 24], cp_spacing_scaler=3.0,
                 smoothing_variance=[2, 1, 0], sampling_rate=[1], neighborhood_sampling=[1],
                 num_function_evaluations=[100, 100, 100], metric="ncc", reg_rd=[1e-3],
                 initial_step_size=[1000.0], tensor_weights=[0])


class ConvDesc(C.Structure):
    _fields_ = [("batch", C.c_int32), ("in_size", C.c_int32 * 3), ("in_channels", C.c_int32),
                ("out_channels", C.c_int32), ("stride", C.c_int32)]

    @classmethod
    def make(cls, batch, in_size, cin, cout, stride):
        d = cls()
        d.batch = batch
        for a in range(3):
            d.in_size[a] = int(in_size[a])
        d.in_channels, d.out_channels, d.stride = cin, cout, stride
        return d


_bound = False


def _lib():
    global _bound
    L = lib()
    if not _bound:
        vp, fp = C.c_void_p, C.POINTER(C.c_float)
        dp = C.POINTER(ConvDesc)
        L.skm_conv3d_out_size.argtypes = [dp, C.POINTER(C.c_int32)]
        L.skm_conv3d_weight_layout.argtypes = [dp] + [C.POINTER(C.c_int32)] * 4
        L.skm_conv3d_pack_weights.argtypes = [dp, vp, vp, vp, vp]
        L.skm_conv3d_forward.argtypes = [dp, vp, vp, vp, C.c_int32, vp, vp, vp, vp]
        L.skm_conv3d_backward_data.argtypes = [dp, vp, vp, vp, vp, vp, vp, vp]
        L.skm_conv3d_backward_weights_workspace.argtypes = [dp]
        L.skm_conv3d_backward_weights_workspace.restype = C.c_size_t
        L.skm_conv3d_backward_weights.argtypes = [dp, vp, vp, vp, vp, vp, C.c_size_t, vp, vp]
        L.skm_adam_step.argtypes = [vp, vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32,
                                    vp]
        L.skm_mse_loss.argtypes = [vp, vp, C.c_int64, vp, vp, vp]
        L.skm_f32_to_bf16.argtypes = [vp, C.c_int64, vp, vp]
        _bound = True
    return L


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def out_size(size, stride):
    return tuple((n - 1) // stride + 1 for n in size)


class ConvLayer:
    """One 3x3x3 convolution: FP32 master weights (C_out, 27 C_in) + bias, packed bf16 operands,
    Adam moments."""

    def __init__(self, torch, cin, cout, stride, relu, rng):
        self.torch, self.cin, self.cout, self.stride, self.relu = torch, cin, cout, stride, relu
        dev = torch.device("cuda")
        std = np.sqrt(2.0 / (27 * cin)) if relu else np.sqrt(1.0 / (27 * cin))
        w = rng.normal(0.0, std, (cout, 27 * cin)).astype(np.float32)
        self.w = torch.tensor(w, device=dev)
        self.b = torch.zeros(cout, dtype=torch.float32, device=dev)
        d = ConvDesc.make(1, (8, 8, 8), cin, cout, stride)
        fr, fl, dr, dl = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(_lib().skm_conv3d_weight_layout(C.byref(d), C.byref(fr), C.byref(fl), C.byref(dr), C.byref(dl)))
        self.wf = torch.zeros((fr.value, fl.value), dtype=torch.bfloat16, device=dev)
        self.wt = torch.zeros((dr.value, dl.value), dtype=torch.bfloat16, device=dev)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)

    def desc(self, batch, in_size):
        return ConvDesc.make(batch, in_size, self.cin, self.cout, self.stride)

    def pack(self, stream):
        d = self.desc(1, (8, 8, 8))
        check(_lib().skm_conv3d_pack_weights(C.byref(d), _p(self.w), _p(self.wf), _p(self.wt), stream))

    def load(self, w, b):
        self.w.copy_(self.torch.tensor(np.asarray(w, np.float32).reshape(self.cout, -1)))
        self.b.copy_(self.torch.tensor(np.asarray(b, np.float32)))


class WarmStartNet:
    """The encoder-decoder on one GPU; forward / backward / Adam through the library's kernels."""

    def __init__(self, seed=0, label_scale=1.0):
        import torch
        self.torch = torch
        rng = np.random.default_rng(seed)
        self.layers = [ConvLayer(torch, ci, co, s, r, rng) for ci, co, s, r in LAYERS]
        self.err = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.label_scale = float(label_scale)
        self.level0_iterations = 0        # first-level iterations after the warm start (validated)
        self.step_count = 0
        self._acts = None
        self.pack()

    def stream(self):
        return C.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def pack(self):
        s = self.stream()
        for L in self.layers:
            L.pack(s)

    def _check_err(self):
        self.torch.cuda.synchronize()
        if int(self.err.item()) != 0:
            self.err.zero_()
            raise RuntimeError("a bounded tensor-core wait gave up in a convolution kernel")

    def forward(self, x):
        """x: bf16 (B, Z, Y, X, 2) on the GPU -> FP32 (B, z, y, x, 3) predictions (scaled labels)."""
        torch = self.torch
        B = x.shape[0]
        size = (x.shape[3], x.shape[2], x.shape[1])
        s = self.stream()
        acts = [x]
        pred = None
        for i, L in enumerate(self.layers):
            osz = out_size(size, L.stride)
            y = torch.empty((B, osz[2], osz[1], osz[0], L.cout), dtype=torch.bfloat16, device="cuda")
            last = i == len(self.layers) - 1
            y32 = torch.empty((B, osz[2], osz[1], osz[0], L.cout), dtype=torch.float32, device="cuda") if last else None
            d = L.desc(B, size)
            check(_lib().skm_conv3d_forward(C.byref(d), _p(acts[-1]), _p(L.wf), _p(L.b), int(L.relu), _p(y), _p(y32),
                                            _p(self.err), s))
            acts.append(y)
            size = osz
            pred = y32
        self._acts = acts
        return pred

    def backward(self, dpred):
        """dpred: bf16 gradient of the loss w.r.t. the predictions; fills every layer's gw, gb."""
        torch = self.torch
        acts = self._acts
        s = self.stream()
        dy = dpred
        for i in range(len(self.layers) - 1, -1, -1):
            L = self.layers[i]
            x = acts[i]
            B = x.shape[0]
            size = (x.shape[3], x.shape[2], x.shape[1])
            d = L.desc(B, size)
            ws = _lib().skm_conv3d_backward_weights_workspace(C.byref(d))
            work = torch.empty(ws, dtype=torch.uint8, device="cuda")
            check(_lib().skm_conv3d_backward_weights(C.byref(d), _p(x), _p(dy), _p(L.gw), _p(L.gb), _p(work), ws,
                                                     _p(self.err), s))
            if i > 0:
                dx = torch.empty_like(x)
                check(_lib().skm_conv3d_backward_data(C.byref(d), _p(dy), _p(L.wt), _p(x), _p(dx), None, _p(self.err),
                                                      s))
                dy = dx

    def train_step(self, x, target, lr=1e-3):
        """One Adam step on the MSE between predictions and (scaled) targets; returns the loss."""
        pred = self.forward(x)
        dpred = self.torch.empty(pred.shape, dtype=self.torch.bfloat16, device="cuda")
        s = self.stream()
        check(_lib().skm_mse_loss(_p(pred), _p(target), pred.numel(), _p(self.loss), _p(dpred), s))
        self.backward(dpred)
        self.step_count += 1
        for L in self.layers:
            check(_lib().skm_adam_step(_p(L.w), _p(L.gw), _p(L.mw), _p(L.vw), L.w.numel(), lr, 0.9, 0.999, 1e-8,
                                       self.step_count, s))
            check(_lib().skm_adam_step(_p(L.b), _p(L.gb), _p(L.mb), _p(L.vb), L.b.numel(), lr, 0.9, 0.999, 1e-8,
                                       self.step_count, s))
        self.pack()
        self._check_err()
        return float(self.loss.item())

    def predict_alpha(self, fixed, moving):
        """Planar kernel weights [3 * C] of the first level from one pair (Z, Y, X) float arrays."""
        x = pair_tensor(self.torch, [(fixed, moving)])
        pred = self.forward(x)
        self._check_err()
        out = pred[0].reshape(-1, 3).double().cpu().numpy() * self.label_scale
        return np.ascontiguousarray(out.T.reshape(-1))

    # ---- persistence
    def save(self, path=WEIGHTS_PATH):
        arrs = {"label_scale": np.array(self.label_scale), "level0_iterations": np.array(self.level0_iterations)}
        for i, L in enumerate(self.layers):
            arrs["w%d" % i] = L.w.cpu().numpy()
            arrs["b%d" % i] = L.b.cpu().numpy()
        np.savez_compressed(path, **arrs)

    @classmethod
    def load(cls, path=WEIGHTS_PATH):
        z = np.load(path)
        net = cls(label_scale=float(z["label_scale"]))
        net.level0_iterations = int(z["level0_iterations"]) if "level0_iterations" in z else 0
        for i, L in enumerate(net.layers):
            L.load(z["w%d" % i], z["b%d" % i])
        net.pack()
        return net


def pair_tensor(torch, pairs):
    """(fixed, moving) arrays (Z, Y, X) -> bf16 (B, Z, Y, X, 2) on the GPU."""
    a = np.stack([np.stack([np.asarray(f, np.float32), np.asarray(m, np.float32)], axis=-1) for f, m in pairs])
    return torch.tensor(a, device="cuda").to(torch.bfloat16).contiguous()


# ---- data: pairs and the plain optimizer's first-level alpha -------------------------------------

def _make_pair(seed):
    from . import synth
    f, m, _ = synth.ellipsoids3d(seed=seed, shape=(INPUT_SIZE[2], INPUT_SIZE[1], INPUT_SIZE[0]))
    return f.astype(np.float32), m.astype(np.float32)


def make_pairs(seeds, workers=None):
    """Seeded config-2-style pairs at 96x96x64 (a process pool started with spawn)."""
    import multiprocessing as mp
    workers = workers or min(len(seeds), os.cpu_count() or 1, 8)     # a few hundred MB of host memory each
    if workers <= 1:
        return [_make_pair(s) for s in seeds]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_make_pair, list(seeds))


def first_level_alpha(fixed, moving):
    """The plain method's converged first-level kernel weights (zero start, 100 iterations)."""
    from . import register as R
    got = {}
    R.register(moving, fixed, (1.0, 1.0, 1.0), None, LEVEL0,
               on_level_parameters=lambda lvl, a: got.__setitem__(lvl, a))
    return got[0]


def train(n_train=256, epochs=40, batch=8, lr=2e-3, seed=0, log=None, pairs=None, labels=None):
    """Generates the data (unless given), trains on the GPU, returns (net, history)."""
    import torch
    seeds = list(range(10_000 + seed * 100_000, 10_000 + seed * 100_000 + n_train))
    t0 = time.perf_counter()
    if pairs is None:
        pairs = make_pairs(seeds)
    if labels is None:
        labels = np.stack([first_level_alpha(f, m) for f, m in pairs])      # (n, 3 C)
    t_data = time.perf_counter() - t0
    scale = float(np.std(labels)) or 1.0
    net = WarmStartNet(seed=seed, label_scale=scale)
    X = pair_tensor(torch, pairs)
    C_ = labels.shape[1] // 3
    # network output (B, z, y, x, 3) with x fastest: [b][j][d] -> labels are planar [b][d][j]
    Y = torch.tensor((labels.reshape(-1, 3, C_).transpose(0, 2, 1) / scale).astype(np.float32), device="cuda")
    grid = tuple(reversed(out_grid(X.shape)))                                # (z, y, x) of the alpha grid
    Y = Y.reshape((len(pairs),) + grid + (3,))
    rng = np.random.default_rng(seed)
    hist = []
    t1 = time.perf_counter()
    for ep in range(epochs):
        order = rng.permutation(len(pairs))
        tot = 0.0
        for k in range(0, len(order) - batch + 1, batch):
            idx = torch.tensor(order[k:k + batch], device="cuda")
            xb = X.index_select(0, idx)
            yb = Y.index_select(0, idx)
            # mirror symmetry: flipping the pair along an axis flips the control-point grid (it is
            # centred on the image) and negates that component of alpha
            for axis in range(3):
                if rng.uniform() < 0.5:
                    xb = xb.flip(3 - axis)
                    yb = yb.flip(3 - axis)
                    yb[..., axis] = -yb[..., axis]
            tot += net.train_step(xb.contiguous(), yb.reshape(batch, -1).contiguous(), lr=lr)
        hist.append(tot / max(1, len(order) // batch))
        if log:
            log("epoch %d loss %.5f" % (ep, hist[-1]))
    return net, {"loss": hist, "data_s": t_data, "train_s": time.perf_counter() - t1, "label_scale": scale,
                 "n_train": len(pairs)}


def out_grid(shape):
    """(x, y, z) size of the network's output for a (B, Z, Y, X, C) input."""
    size = (shape[3], shape[2], shape[1])
    for _, _, s, _ in LAYERS:
        size = out_size(size, s)
    return size


def choose_level0_iterations(net, seeds, candidates=(0, 10, 25, 50), config=None):
    """The fewest first-level iterations after the warm start with which every validation pair
    reaches the plain run's final NCC within 1e-3 (the plain schedule's count if none does)."""
    from . import register as R
    cfg = dict(config or MS_CONFIG)
    pairs = make_pairs(seeds, workers=1)
    plain = [final_ncc(f, m, R.register(m, f, (1.0, 1.0, 1.0), None, cfg)[0]) for f, m in pairs]
    for k in candidates:
        ok = True
        for (f, m), p in zip(pairs, plain):
            d, _, used = register_with_warm_start(net, f, m, cfg, level0_iterations=k)
            if final_ncc(f, m, d) < p - 1e-3:
                ok = False
                break
        if ok:
            return k
    return int(cfg["num_function_evaluations"][0])


def register_with_warm_start(net, fixed, moving, config=None, level0_iterations=None):
    """Multi-scale registration of `moving` onto `fixed` starting the first level from the network's
    prediction (that level then runs `level0_iterations` iterations, the later levels their plain
    schedule); falls back to the plain zero start when the prediction does not lower the first
    level's metric value.  Returns (displacement, report, used_warm_start)."""
    from . import register as R
    cfg = dict(config or MS_CONFIG)
    alpha = net.predict_alpha(fixed, moving)
    v_warm, v_zero = first_level_values(fixed, moving, [alpha, np.zeros_like(alpha)])
    if not v_warm < v_zero:
        disp, rep = R.register(moving, fixed, (1.0, 1.0, 1.0), None, cfg)       # fallback: the plain method
        return disp, rep, False
    its = list(cfg["num_function_evaluations"])
    its[0] = net.level0_iterations if level0_iterations is None else level0_iterations
    disp, rep = R.register(moving, fixed, (1.0, 1.0, 1.0), None, dict(cfg, num_function_evaluations=its),
                           first_level_parameters=alpha)
    return disp, rep, True


def first_level_values(fixed, moving, alphas):
    """Metric values (NCC + RD) of the first level at each planar kernel-weight vector: the same
    preprocessing as skm_register's first level (threshold + rescale, smoothing variance 2,
    B-spline prefilter, control spacing float(48) / 3 = 16 voxels)."""
    from . import register as R
    from .abi import MetricDesc
    from .evaluator import GpuKernelEvaluator, bspline_coefficients
    from .problem import Problem
    th = (-1500, 3500)
    f = R.gaussian_smooth(R.threshold_rescale(fixed, th), (1.0, 1.0, 1.0), float(LEVEL0["smoothing_variance"][0]))
    m = R.gaussian_smooth(R.threshold_rescale(moving, th), (1.0, 1.0, 1.0), float(LEVEL0["smoothing_variance"][0]))
    s4, s0 = float(LEVEL0["sigma_C4"][0]), float(LEVEL0["sigma_C0"][0])
    cps = float(np.float32(min(s4, s0)) / np.float32(LEVEL0["cp_spacing_scaler"]))
    pb = Problem(fixed=f, moving_coefficients=bspline_coefficients(m), spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                 sigma_c0=s0, sigma_c4=s4, cp_spacing=cps)
    ev = GpuKernelEvaluator(pb)
    m = MetricDesc.make("ncc", rd=float(LEVEL0["reg_rd"][0]))
    out = [ev.metric(m, a, np.ones(pb.C), derivative=False)[0]["value"] for a in alphas]
    ev.close()
    return out


def evaluate_gain(net, seeds, config=None):
    """Held-out pairs: the plain multi-scale registration (zero start) against the warm-started one.
    Per pair: wall time, optimizer iterations and final NCC of both (NCC of the rescaled pair warped
    by the summed field, every voxel); `within_1e-3`: the warm start reaches the plain final NCC
    within 1e-3."""
    from . import register as R
    cfg = dict(config or MS_CONFIG)
    pairs = make_pairs(seeds, workers=1)
    R.register(pairs[0][1][::4, ::4, ::4].copy(), pairs[0][0][::4, ::4, ::4].copy(), (1.0, 1.0, 1.0), None,
               dict(cfg, num_function_evaluations=[2]))                 # warm-up of the library
    out = []
    for (f, m), s in zip(pairs, seeds):
        t0 = time.perf_counter()
        d_plain, rep_p = R.register(m, f, (1.0, 1.0, 1.0), None, cfg)
        t_plain = time.perf_counter() - t0
        t0 = time.perf_counter()
        d_warm, rep_w, used = register_with_warm_start(net, f, m, cfg)
        t_warm = time.perf_counter() - t0
        n_p, n_w = final_ncc(f, m, d_plain), final_ncc(f, m, d_warm)
        out.append({"seed": int(s), "plain_s": t_plain, "warm_s": t_warm, "plain_iterations": int(sum(rep_p["iterations"])),
                    "warm_iterations": int(sum(rep_w["iterations"])), "plain_ncc": n_p, "warm_ncc": n_w,
                    "used_warm_start": bool(used), "within_1e-3": bool(n_w >= n_p - 1e-3),
                    "speedup": t_plain / t_warm})
    return out


def final_ncc(fixed, moving, disp):
    """NCC (positive) of the rescaled pair, moving warped by `disp`, every voxel sampled."""
    from . import register as R
    from .evaluator import GpuKernelEvaluator, bspline_coefficients
    from .problem import Problem
    f = R.threshold_rescale(fixed, (-1500, 3500))
    m = R.threshold_rescale(moving, (-1500, 3500))
    pb = Problem(fixed=f, moving_coefficients=bspline_coefficients(m), spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                 sigma_c0=24.0, sigma_c4=12.0, cp_spacing=4.0)
    ev = GpuKernelEvaluator(pb)
    r = ev.getValue(GpuKernelEvaluator.NCC, np.zeros((pb.C, pb.D)), np.ones(pb.C),
                    np.ascontiguousarray(disp.reshape(-1, f.ndim)))
    ev.close()
    return -float(r["measure"])


def time_steps(batch=8, steps=20):
    """Training steps on seeded random 96x96x64 inputs (no data generation): milliseconds per step,
    the forward + backward + Adam of the whole network on the library's kernels."""
    import torch
    rng = np.random.default_rng(0)
    net = WarmStartNet(seed=0)
    x = torch.tensor(rng.uniform(size=(batch, INPUT_SIZE[2], INPUT_SIZE[1], INPUT_SIZE[0], 2)).astype(np.float32),
                     device="cuda").to(torch.bfloat16).contiguous()
    g = out_grid(x.shape)
    y = torch.tensor(rng.normal(size=(batch, g[0] * g[1] * g[2] * 3)).astype(np.float32), device="cuda")
    for _ in range(3):
        net.train_step(x, y)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        net.train_step(x, y)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / steps * 1e3
    flops = 0.0
    size = (INPUT_SIZE[0], INPUT_SIZE[1], INPUT_SIZE[2])
    for ci, co, s, _ in LAYERS:
        o = out_size(size, s)
        flops += 2.0 * batch * o[0] * o[1] * o[2] * co * 27 * ci * 3          # forward, data and weight grads
        size = o
    return {"batch": batch, "ms_per_step": ms, "tflops": flops / (ms * 1e-3) / 1e12, "steps": steps}


def main(argv=None):
    """python -m skmimageregistration_b200.warmstart train [--n N] [--epochs E] [--out PATH]"""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("command", choices=["train", "gain", "steps"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--weights", default=WEIGHTS_PATH)
    ap.add_argument("--held-out", type=int, default=4)
    ap.add_argument("--validation", type=int, default=6)
    a = ap.parse_args(argv)
    if a.command == "train":
        net, hist = train(n_train=a.n, epochs=a.epochs, batch=a.batch, lr=a.lr, log=print)
        net.level0_iterations = choose_level0_iterations(net, list(range(800_000, 800_000 + a.validation)))
        hist["level0_iterations"] = net.level0_iterations
        net.save(a.out)
        print(json.dumps({k: v for k, v in hist.items()}))
    elif a.command == "steps":
        print(json.dumps(time_steps(batch=a.batch, steps=a.epochs)))
    else:
        net = WarmStartNet.load(a.weights)
        print(json.dumps(evaluate_gain(net, list(range(900_000, 900_000 + a.held_out)))))


if __name__ == "__main__":
    main()
