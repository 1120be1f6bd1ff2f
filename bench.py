#!/usr/bin/env python
"""Benchmark: SKM optimizer iterations per second on one or more B200s.

One step = one iteration of the adaptive-step gradient-descent optimizer on the
``ncc128`` workload (128x128x96 pair, 24,576 control points, kernel support 12
voxels, NCC + RD regularizer 1e-3, every voxel sampled): transform + B-spline warp +
NCC statistics + control-point derivative + regularizer + parameter update.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* ``value``: device-resident loop (parameters and optimizer state stay in HBM, one CUDA
  graph per iteration); each timed iteration is bracketed by CUDA events on the
  evaluator's stream, with an L2 flush (256 MB write) before every iteration outside
  the events.  N > 1: one independent pair per GPU (weak scaling), value = all
  iterations / slowest rank's time.
* ``e2e``: the reference-facing C-ABI call with host buffers, the way the ITK glue
  drives it: per step the planar parameters and weights go host->device, value and
  derivative come back device->host, and the optimizer update runs on the host.
* ``cpu_baseline`` / ``--impl reference``: the FP64 CPU restatement of the same
  evaluation (oracle/, OpenMP over all host cores); the reference itself has no CPU
  implementation of this path.  The reference arm additionally times the reference's
  own CUDA evaluator (built from its sources for sm_100a) when it is available.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ncc128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-multiscale", action="store_true",
                    help="skip the multi-scale registration comparison (s/pair)")
    ap.add_argument("--gemm", default="auto", choices=["auto", "cuda"],
                    help="table-path GEMMs: auto = tensor cores where they fit, cuda = CUDA-core kernels")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0: same as --steps (capped at 300)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-pair batched line (config 4)")
    ap.add_argument("--no-ct3d", action="store_true", help="skip the CT-like LCC line (config 3)")
    ap.add_argument("--only", default="all", choices=["all", "batch", "ct3d", "ncc128", "mse2d"],
                    help="run one secondary measurement alone and print its JSON (batch: --batch-pairs pairs)")
    ap.add_argument("--batch-pairs", type=int, default=64)
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def measured_peaks():
    try:
        with open(PEAKS_PATH) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def fp32_peak_tflops(torch):
    """CUDA-core FP32 peak measured live: cuBLAS SGEMM 8192^3 with TF32 off, best of 5."""
    torch.backends.cuda.matmul.allow_tf32 = False
    torch.backends.cudnn.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    best = None
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e)
        best = ms if best is None else min(best, ms)
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def tf32_peak_tflops(torch):
    """Tensor-core TF32 peak measured live: cuBLAS FP32 GEMM 8192^3 with TF32 allowed, best of 5."""
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    best = None
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        ms = s.elapsed_time(e)
        best = ms if best is None else min(best, ms)
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = False
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def pair_count(pb):
    """(fixed texel, control point) pairs inside the forward box (separable per axis)."""
    tot = 1
    support = min(pb.sigma_c4, pb.sigma_c0)
    for d in range(pb.D):
        n = pb.size[d]
        idx = np.arange(n)
        p = pb.origin[d] + pb.spacing[d] * idx
        ip = (p - pb.cp_origin[d]) / pb.cp_sp[d]
        sh = support / pb.cp_sp[d]
        lo = np.clip(np.trunc(ip - sh + 1.0), 0, pb.cp_size[d] - 1)
        hi = np.clip(np.trunc(ip + sh), 0, pb.cp_size[d] - 1)
        tot *= int((hi - lo + 1).sum())
    return tot


def fused_basis(pb):
    """Algorithmic HBM bytes and FLOPs of one iteration on the fused basis: per fixed voxel the fixed
    value and one moving-image coefficient (8 B), per control point alpha + weight read (16 B) and
    the derivative written (12 B); FLOPs of the direct formulation, 22 FLOP per kernel evaluation
    + 7 (value pass) and + 6m + 1 (derivative pass, m = 1 MSE, 2 NCC) per (voxel, control point)
    pair in support, plus the 4^D-tap B-spline value and gradient per voxel."""
    N, C, D = pb.n_texels, pb.C, pb.D
    pairs = pair_count(pb)
    return {"voxel_bytes": 8.0 * N, "cp_bytes": 28.0 * C, "bytes": 8.0 * N + 28.0 * C,
            "pairs": pairs, "flops_direct": pairs * (29.0 + 35.0) + N * (2 * 4 ** D * 2 + 2 * 4 ** (D - 1) * 3)}


def kernel_work(pb, info, phases):
    """Per-kernel executed work (FLOPs) and algorithmic bytes of one iteration, with its time.

    Two byte counts per kernel: "bytes" counts what the kernel split reads and writes, the
    intermediates between kernels included (u, the (grad M, m) records, the Contrib array);
    "alg_bytes" counts only the fused basis (fused_basis): the warp kernel's fixed value and moving
    coefficient per voxel, the transform's alpha + weight and the gather's derivative per control
    point; the contrib GEMM has none (everything it touches is an intermediate).

    Table path: the transform and the contrib GEMM each need 3 FMAs per (cell, phase, tap)
    triple (algorithmic FLOPs); on the tensor cores (path 3) they execute, per tile of 128
    (component, cell) rows, MMAs of N x K with N = 1.5 x tc_transform_n (hi x [hi; lo] and lo x hi)
    and 3 x tc_contrib_n (hi hi, hi lo, lo hi) -- "tensor_flops".  The warp kernel evaluates a
    4^D-tap B-spline with gradient per texel; the gather adds 3 values per (control point, tap).
    Bytes count every input once and every output once.
    Generic path: one kernel evaluation (22 FLOP) per (texel, control point) pair in support.
    """
    D = pb.D
    N, C = pb.n_texels, pb.C
    ncoef = pb.moving_coefficients.size
    taps_b = 4 ** D
    bspline_flops = N * (2 * taps_b * 2 + 2 * (taps_b // 4) * 3)
    if info["path"] in (2, 3):
        cells, nph, ntap = info["table_cells"], info["table_phases"], info["table_taps"]
        gemm = 2.0 * D * cells * nph * ntap
        tc = info["path"] == 3
        tr = {"name": "table_transform_tc_kernel" if tc else "table_transform_kernel",
              "bound": "tensor" if tc else "fp32", "ms": phases["transform"],
              "flops": gemm, "bytes": C * 16 + nph * ntap * 4 + cells * nph * 4 * D}
        # contributions: one per (cell, tap with a nonzero table column) -- the tensor-core path
        # skips the all-zero taps, the CUDA-core one stores every tap of the box
        ctaps = (info.get("tc_contrib_taps") or ntap) if tc else ntap
        co = {"name": "table_contrib_tc_kernel" if tc else "table_contrib_kernel",
              "bound": "tensor" if tc else "fp32", "ms": phases["contrib"], "flops": gemm,
              "bytes": cells * nph * (16 + 4) + nph * ntap * 4 + D * ctaps * cells * 4}
        if tc:
            tr["tensor_flops"] = (2.0 * 128 * 1.5 * info["tc_transform_n"] * info["tc_transform_k"]
                                  * info["tc_transform_tiles"])
            co["tensor_flops"] = (2.0 * 128 * 3 * info["tc_contrib_n"] * info["tc_contrib_k"]
                                  * info["tc_contrib_tiles"])
        tr["alg_bytes"] = 16.0 * C
        co["alg_bytes"] = 0.0
        return {
            "transform": tr,
            "warp": {"name": "table_warp_tma_kernel" if info.get("warp_staged") else "table_warp_kernel",
                     "bound": "hbm", "ms": phases["warp"], "flops": bspline_flops,
                     "bytes": cells * nph * (4 * D + 4 + 16) + ncoef * 4, "alg_bytes": 8.0 * N},
            "contrib": co,
            "gather": {"name": "table_gather_rows_kernel", "bound": "hbm", "ms": phases["gather"],
                       "flops": 3.0 * C * ntap + 20.0 * C * info["table_regularizer_offsets"],
                       "bytes": 3 * ctaps * cells * 4 + C * 16 + C * D * 8, "alg_bytes": 12.0 * C},
        }
    pairs = pair_count(pb)
    return {
        "value": {"name": "value_kernel", "bound": "fp32", "ms": phases["transform"], "flops": pairs * 29.0 + bspline_flops,
                  "bytes": N * 4 + ncoef * 4 + C * 16 + N * 16, "alg_bytes": 8.0 * N + 16.0 * C},
        "derivative": {"name": "derivative_kernel", "bound": "fp32", "ms": phases["gather"], "flops": pairs * 35.0,
                       "bytes": N * 20 + C * 16 + C * D * 8, "alg_bytes": 12.0 * C},
    }


def iteration_roofline(pb, ms_step, hbm_peak, hbm_src, fp32_peak):
    """The whole optimizer iteration against both roofs on the fused basis (fused_basis)."""
    fb = fused_basis(pb)
    gbs = fb["bytes"] / (ms_step * 1e-3) / 1e9
    tflops = fb["flops_direct"] / (ms_step * 1e-3) / 1e12
    return {"ms": ms_step, "algorithmic_bytes": fb["bytes"], "achieved_gbs": gbs, "hbm_peak_gbs": hbm_peak,
            "hbm_frac": gbs / hbm_peak, "hbm_peak_source": hbm_src, "flops_direct_formulation": fb["flops_direct"],
            "pairs_per_pass": fb["pairs"], "fp32_equivalent_tflops": tflops, "fp32_peak_tflops": fp32_peak,
            "fp32_frac": tflops / fp32_peak,
            "note": "bytes: 8 B per fixed voxel + 28 B per control point; FLOPs: direct formulation "
                    "(every kernel value evaluated), which the phase table replaces by table reads"}


# ------------------------------------------------------------------------------------------------
def cpu_port_rate(pb, mdesc, budget_s=20.0, max_steps=5, min_steps=1, threads=None):
    """FP64 CPU restatement: full-size metric evaluations + host update, steps/s."""
    from oracle import oracle as O
    threads = threads or os.cpu_count()
    O.set_num_threads(threads)
    orc = O.Oracle(pb)
    P = pb.num_parameters
    params = np.zeros(P)
    cpw = np.ones(pb.C)
    steps = 0
    t0 = time.perf_counter()
    while True:
        _, g = orc.metric(mdesc, params, cpw)
        params = params + 1e-3 * g
        steps += 1
        el = time.perf_counter() - t0
        if steps >= max_steps or (steps >= min_steps and el >= budget_s):
            break
    return steps / el, steps, el, threads


def reference_cuda_rate(pb, mdesc, budget_s=20.0, max_steps=50):
    """The reference's own GpuKernelEvaluator (oracle/_ref, double build), driven like its ITK glue."""
    from oracle import oracle as O
    path = O.ref_gpu_path(pb.D, True)
    if not os.path.exists(path):
        return None
    ref = O.RefGpu(pb, double=True)
    ref.set_regularizers(mdesc.reg_rkhs, mdesc.reg_rd, mdesc.reg_rd_scaling, mdesc.reg_pg, mdesc.reg_pg_scaling)
    P = pb.num_parameters
    cp = np.zeros((pb.C, pb.D))
    cpw = np.ones(pb.C)
    ref.evaluate(mdesc.metric, cp, cpw)                     # warm-up
    steps = 0
    t0 = time.perf_counter()
    while True:
        _, g = ref.evaluate(mdesc.metric, cp, cpw)
        cp = cp - 1e-3 * g.reshape(pb.D, -1).T                # negated gradient step (metric hxx:528)
        steps += 1
        el = time.perf_counter() - t0
        if steps >= max_steps or el >= budget_s:
            break
    ref.close()
    return steps / el, steps, el


# ------------------------------------------------------------------------------------------------
# ------------------------------------------------------------------------------------------------
# multi-scale registration of the ncc128 pair: ours (skm_register) against the same scale loop
# driven by the reference's own GpuKernelEvaluator (host optimizer loop as in the ITK glue,
# reference B-spline prefilter compiled for the host, FP64 smoothing / threshold restatements
# standing in for the ITK filters)
MS_CONFIG = dict(num_scales=3, sigma_C4=[48, 24, 12], sigma_C0=[96, 48, 24], cp_spacing_scaler=3.0,
                 smoothing_variance=[2, 1, 0], sampling_rate=[1], neighborhood_sampling=[1],
                 num_function_evaluations=[100, 100, 100], metric="ncc", reg_rd=[1e-3],
                 initial_step_size=[1000.0], tensor_weights=[0])


def final_ncc(fixed, moving, disp, spacing):
    """NCC of the rescaled pair with the moving image warped by `disp` (our evaluator, subsample 1)."""
    from skmimageregistration_b200 import register as R
    from skmimageregistration_b200.evaluator import GpuKernelEvaluator, bspline_coefficients
    from skmimageregistration_b200.problem import Problem
    f = R.threshold_rescale(fixed, MS_CONFIG.get("intensity_thresholds", (-1500, 3500)))
    m = R.threshold_rescale(moving, MS_CONFIG.get("intensity_thresholds", (-1500, 3500)))
    pb = Problem(fixed=f, moving_coefficients=bspline_coefficients(m), spacing=spacing, origin=(0.0,) * f.ndim,
                 sigma_c0=24.0, sigma_c4=12.0, cp_spacing=4.0)
    ev = GpuKernelEvaluator(pb)
    r = ev.getValue(GpuKernelEvaluator.NCC, np.zeros((pb.C, pb.D)), np.ones(pb.C),
                    np.ascontiguousarray(disp.reshape(-1, f.ndim)))
    ev.close()
    return -float(r["measure"])


def reference_multiscale(fixed, moving, spacing, config):
    """The scale loop with the reference's GpuKernelEvaluator; returns (displacement, seconds)."""
    from oracle import multiscale as M
    from oracle import oracle as O
    from skmimageregistration_b200.problem import Problem
    from skmimageregistration_b200.register import current, full_config
    c = full_config(config)
    D = fixed.ndim
    host = O.ref_host(D)
    t0 = time.perf_counter()
    th = c.get("intensity_thresholds") or []
    ref = M.threshold_rescale(moving, th if len(th) == 2 else None)
    tar = M.threshold_rescale(fixed, th if len(th) == 2 else None)
    past = None
    for s in range(int(c["num_scales"])):
        var = float(current(c, "smoothing_variance", s))
        ref_s = M.gaussian_smooth(ref, spacing, var) if var > 1e-5 else ref
        tar_s = M.gaussian_smooth(tar, spacing, var) if var > 1e-5 else tar
        coeffs = np.zeros(tuple(n + 3 for n in ref_s.shape))
        size = (C.c_int32 * 3)(*(list(reversed(ref_s.shape)) + [1] * (3 - D)))
        host.skmref_bspline_coefficients(size, ref_s.ctypes.data_as(C.POINTER(C.c_double)),
                                         coeffs.ctypes.data_as(C.POINTER(C.c_double)))
        s4, s0 = float(current(c, "sigma_C4", s)), float(current(c, "sigma_C0", s))
        cps = float(np.float32(min(s4, s0)) / np.float32(c["cp_spacing_scaler"]))
        pb = Problem(fixed=tar_s, moving_coefficients=coeffs, spacing=spacing, origin=(0.0,) * D, sigma_c0=s0,
                     sigma_c4=s4, cp_spacing=cps, subsample=int(current(c, "sampling_rate", s)),
                     subsample_neighborhood=int(current(c, "neighborhood_sampling", s)))
        rg = O.RefGpu(pb, double=True)
        w_rd = float(current(c, "reg_rd", s))
        w_l1 = float(current(c, "reg_l1", s))
        rg.set_regularizers(0.0, w_rd, float(current(c, "reg_rd_scaling", s)), 0.0, 1.0)
        metric = {"mse": 0, "ncc": 1, "lcc": 2}[c["metric"]]
        a, n_it = float(current(c, "initial_step_size", s)), int(current(c, "num_function_evaluations", s))
        orthant = w_l1 > 0 and w_rd <= 0                 # SKMReg.cxx:392-411: L1 as the only regularizer
        P, Cn = pb.num_parameters, pb.C
        pos, base, prev, best = np.zeros(P), np.zeros(P), np.zeros(P), np.zeros(P)
        t_sim, best_v, cpw = 0.0, np.inf, np.ones(Cn)
        dfg = pb.fixed_geometry() if past is not None else None
        for _ in range(n_it):                            # the ITK v4 loop with the adaptive step
            r, g = rg.evaluate(metric, pos.reshape(D, Cn).T, cpw, past, dfg)
            value = r["measure"] + w_rd * r["reg_value_rd"]
            if w_l1 > 0:                                 # host L1 term (itkRegularizedImageToImageMetricv4.hxx:447-466)
                value += w_l1 * float(np.abs(pos).sum())
                nz = pos != 0.0
                g = np.where(nz, g + w_l1 * np.sign(pos),
                             np.where(g < -w_l1, g + w_l1, np.where(g > w_l1, g - w_l1, 0.0)))
            g = -g
            lr = a / (20.0 + t_sim + 1.0)
            sp = float(np.dot(g, prev))
            prev = g
            pos = base + g * lr
            if orthant:
                pos = np.where(pos * base < 0.0, 0.0, pos)
            base = pos
            t_sim = max(0.0, t_sim - 1e6 + (1e7 + 1e6) / (1.0 + 10.0 * math.exp(min(sp, 700.0))))
            if value < best_v:
                best_v, best = value, pos.copy()
        past = rg.displacement_field(np.ascontiguousarray(best.reshape(D, Cn).T), cpw, past, dfg)
        past = np.ascontiguousarray(past.reshape(fixed.shape + (D,)))
        rg.close()
    return past, time.perf_counter() - t0


# config 1: the 2-D 256x256 blob pair, MSE + L1 1e-3, control spacing 8 px and support 16 px at the
# finest of 3 levels, 100 iterations each
MS_CONFIG_2D = dict(num_scales=3, sigma_C4=[64, 32, 16], sigma_C0=[128, 64, 32], cp_spacing_scaler=2.0,
                    smoothing_variance=[2, 1, 0], sampling_rate=[1], neighborhood_sampling=[1],
                    num_function_evaluations=[100, 100, 100], metric="mse", reg_l1=[1e-3], reg_rd=[0.0],
                    initial_step_size=[1000.0], tensor_weights=[0])


def final_mse(fixed, moving, disp, spacing):
    """MSE of the rescaled 2-D pair with the moving image warped by `disp` (our evaluator)."""
    from skmimageregistration_b200 import register as R
    from skmimageregistration_b200.evaluator import GpuKernelEvaluator, bspline_coefficients
    from skmimageregistration_b200.problem import Problem
    f = R.threshold_rescale(fixed, (-1500, 3500))
    m = R.threshold_rescale(moving, (-1500, 3500))
    pb = Problem(fixed=f, moving_coefficients=bspline_coefficients(m), spacing=spacing, origin=(0.0,) * f.ndim,
                 sigma_c0=32.0, sigma_c4=16.0, cp_spacing=8.0)
    ev = GpuKernelEvaluator(pb)
    r = ev.getValue(GpuKernelEvaluator.MSE, np.zeros((pb.C, pb.D)), np.ones(pb.C),
                    np.ascontiguousarray(disp.reshape(-1, f.ndim)))
    ev.close()
    return float(r["measure"])


def multiscale_compare(name="ncc128", override=None):
    """s/pair of the multi-scale registration for both drivers and the final metric each reaches:
    ncc128 (3-D, NCC + RD, the headline) or mse2d (config 1: 2-D 256^2, MSE + L1)."""
    from skmimageregistration_b200 import register as R
    from skmimageregistration_b200 import synth
    if name == "ncc128":
        fixed, moving, _ = synth.ellipsoids3d(seed=0, shape=(96, 128, 128))
        spacing, cfg, volume = (1.0, 1.0, 1.0), MS_CONFIG, "128x128x96"
        score, key, better = final_ncc, "ncc", (lambda a, b: a >= b - 1e-3)
        R.register(moving, fixed, spacing, None, MS_CONFIG)                  # warm-up: one untimed run
    else:
        fixed, moving, _ = synth.blobs2d(seed=0, shape=(256, 256))
        spacing, cfg, volume = (1.0, 1.0), dict(MS_CONFIG_2D, **(override or {})), "256x256"
        score, key, better = final_mse, "mse", (lambda a, b: a <= b + 1e-3 * abs(b))
        R.register(moving, fixed, spacing, None, cfg)                        # warm-up: one untimed run
    # the warm-up above ran the same registration once, untimed (first launches, the memory pool);
    # five timed runs, the median reported, every run's level times (whole level, and the optimizer
    # iterations alone) kept beside it
    runs, run_levels, run_opt = [], [], []
    for _ in range(5):
        t0 = time.perf_counter()
        disp, rep = R.register(moving, fixed, spacing, None, cfg)
        runs.append(time.perf_counter() - t0)
        run_levels.append([round(x, 4) for x in rep["seconds"][:rep["levels_done"]]])
        run_opt.append([round(x, 4) for x in rep["optimize_seconds"][:rep["levels_done"]]])
    ours_s = sorted(runs)[len(runs) // 2]
    out = {"config": dict(cfg, volume=volume), "ours_s_per_pair": ours_s, "ours_runs_s": runs,
           "ours_runs_level_seconds": run_levels, "ours_runs_level_optimize_seconds": run_opt,
           "ours_final_" + key: score(fixed, moving, disp, spacing),
           key + "_before": score(fixed, moving, 0 * disp, spacing), "ours_levels": rep}
    from oracle import oracle as O  # noqa: F401  (reference arm: needs the reference build)
    if os.path.exists(O.ref_gpu_path(fixed.ndim, True)):
        disp_r, ref_s = reference_multiscale(fixed, moving, spacing, cfg)
        out["reference_s_per_pair"] = ref_s
        out["reference_final_" + key] = score(fixed, moving, disp_r, spacing)
        ok = bool(better(out["ours_final_" + key], out["reference_final_" + key]))
        out["matches_reference_final_value"] = ok
        out["s_per_pair_to_reference_" + key] = ours_s if ok else None
        out["speedup"] = ref_s / ours_s
    return out


# config 3: CT-like 256x256x160 volume, 1.5 mm voxels, LCC in the reference's form (window = kernel
# support, radial weight, neighbourhood stride), anisotropic kernels from the structure tensor of each
# level's smoothed target, RKHS + L1, 4 levels down to a 4-voxel control spacing (64x64x40 points)
# The reference-form LCC costs (control points) x (samples in a point's support box) x (window
# neighbours), both of the latter growing with the support cubed; the sampling rates and window
# strides grow with the support (as SKMReg's defaults do, include/ConfigUtils.h) so that every level
# keeps about 70 samples per box and 50 neighbours per window.
CT3D_CONFIG = dict(num_scales=4, sigma_C4=[144, 72, 36, 18], sigma_C0=[288, 144, 72, 36], cp_spacing_scaler=3.0,
                   smoothing_variance=[4, 2, 1, 0], sampling_rate=[64, 32, 16, 8],
                   neighborhood_sampling=[96, 48, 24, 12], num_function_evaluations=[100], metric="lcc",
                   reg_rkhs=[1e-3], reg_l1=[1e-3], initial_step_size=[100.0], tensor_weights=[400, 200, 100, 50])


def ct3d_compare(torch, budget_s=150.0):
    """Config 3 per level, within a time budget: our device optimizer's iterations/s (one warm-up
    iteration, then up to 5 timed ones or 2 s), one evaluation of the reference's GpuKernelEvaluator on
    the same level problem (while the budget lasts) for its iterations/s and for parity (value and
    derivative at alpha = 0, same PCG32 sample shifts), and s/pair = sum over the levels of 100
    iterations / iterations per second.  Every level runs without an earlier level's field (the
    per-iteration cost does not depend on it)."""
    from oracle import oracle as O
    from skmimageregistration_b200 import register as R
    from skmimageregistration_b200 import synth
    from skmimageregistration_b200.abi import MetricDesc, OptimizerDesc
    from skmimageregistration_b200.evaluator import GpuKernelEvaluator, Optimizer, bspline_coefficients
    from skmimageregistration_b200.problem import Problem
    from skmimageregistration_b200.register import current, full_config
    t_start = time.perf_counter()
    fixed, moving, _ = synth.ct3d(seed=0, shape=(160, 256, 256))
    spacing = (1.5, 1.5, 1.5)
    c = full_config(CT3D_CONFIG)
    tar = R.threshold_rescale(fixed, (-1500, 3500))
    ref_img = R.threshold_rescale(moving, (-1500, 3500))
    have_ref = os.path.exists(O.ref_gpu_path(3, True))
    levels, ours_total, ref_total, prev = [], 0.0, 0.0, None
    for s in range(int(c["num_scales"])):
        var = float(current(c, "smoothing_variance", s))
        tar_s = R.gaussian_smooth(tar, spacing, var) if var > 1e-5 else tar
        ref_s = R.gaussian_smooth(ref_img, spacing, var) if var > 1e-5 else ref_img
        s4, s0 = float(current(c, "sigma_C4", s)), float(current(c, "sigma_C0", s))
        cov, tilt = R.anisotropic_tensor(tar_s, spacing, float(np.float32(s4)), float(current(c, "tensor_weights", s)), 2)
        cps = float(np.float32(min(s4, s0)) / np.float32(c["cp_spacing_scaler"]))
        pb = Problem(fixed=tar_s, moving_coefficients=bspline_coefficients(ref_s), spacing=spacing, origin=(0.0,) * 3,
                     sigma_c0=s0, sigma_c4=s4, cp_spacing=cps, subsample=int(current(c, "sampling_rate", s)),
                     subsample_neighborhood=int(current(c, "neighborhood_sampling", s)), weight_tensor=cov,
                     maximum_weight=tilt if tilt >= 0 else 1.0, maximum_eigenvalue_covariance=np.eye(3))
        m = MetricDesc.make("lcc", rkhs=float(current(c, "reg_rkhs", s)), l1=float(current(c, "reg_l1", s)))
        zeros, ones = np.zeros(pb.num_parameters), np.ones(pb.C)
        ev = GpuKernelEvaluator(pb)
        opt = Optimizer(ev, OptimizerDesc.make(a=float(current(c, "initial_step_size", s)), number_of_iterations=1000),
                        m, zeros, ones)
        opt.run(1)
        torch.cuda.synchronize()
        k, t0 = 0, time.perf_counter()
        while k < 5 and (k == 0 or time.perf_counter() - t0 < 2.0):
            opt.run(1)
            k += 1
        ours_it_s = k / (time.perf_counter() - t0)
        opt.close()
        ev.close()
        lv = {"level": s, "control_points": pb.C, "control_spacing_mm": cps, "samples": int(np.prod(
            [n // pb.subsample for n in pb.size])), "tilt": tilt, "ours_iterations_timed": k,
            "ours_iterations_per_s": ours_it_s}
        ours_total += 100.0 / ours_it_s
        # the reference's evaluation costs about (ours) x (taps per neighbour, constant over the
        # levels): its next time is predicted from the last one and run only if it fits the budget
        pred_ref = None if prev is None else prev[1] * prev[0] / ours_it_s
        lv["reference_predicted_s"] = pred_ref
        fits = pred_ref is None or time.perf_counter() - t_start + pred_ref < budget_s
        if have_ref and fits and time.perf_counter() - t_start < budget_s:
            e2 = GpuKernelEvaluator(pb)
            e2.SetRegularizerRKHS(float(current(c, "reg_rkhs", s)))
            r, g = e2.getValueAndDerivative(GpuKernelEvaluator.LCC, np.zeros((pb.C, 3)), ones)
            e2.close()
            rg = O.RefGpu(pb, double=True)
            rg.set_regularizers(rkhs=float(current(c, "reg_rkhs", s)))
            t0 = time.perf_counter()
            rr, gr = rg.evaluate(2, np.zeros((pb.C, 3)), ones)
            t_ref = time.perf_counter() - t0
            rg.close()
            def parity(rr, gr):
                return {"measure_rel": abs(r["measure"] - rr["measure"]) / max(abs(rr["measure"]), 1e-300),
                        "pixels_equal": bool(r["num_pixels_counted"] == rr["num_pixels_counted"]),
                        "derivative_max_rel": float(np.max(np.abs(g - gr)) / max(np.max(np.abs(gr)), 1e-300))}
            lv.update(reference_iterations_per_s=1.0 / t_ref, parity=parity(rr, gr))
            if os.path.exists(O.ref_gpu_path(3, True, ieee=True)):
                # the same reference sources built with IEEE arithmetic (no fast math, no contraction)
                ri = O.RefGpu(pb, double=True, ieee=True)
                ri.set_regularizers(rkhs=float(current(c, "reg_rkhs", s)))
                rri, gri = ri.evaluate(2, np.zeros((pb.C, 3)), ones)
                ri.close()
                lv["parity_ieee_build"] = parity(rri, gri)
                lv["reference_builds"] = {
                    "measure_rel": abs(rr["measure"] - rri["measure"]) / max(abs(rri["measure"]), 1e-300),
                    "derivative_max_rel": float(np.max(np.abs(gr - gri)) / max(np.max(np.abs(gri)), 1e-300))}
            ref_total += 100.0 * t_ref
            prev = (ours_it_s, t_ref)
        else:
            lv["reference_iterations_per_s"] = None
            ref_total = None if not have_ref else ref_total
        levels.append(lv)
    out = {"config": dict(CT3D_CONFIG, volume="256x256x160", spacing_mm=1.5), "levels": levels,
           "ours_s_per_pair_estimate": ours_total,
           "reference_s_per_pair_estimate": ref_total if all(l["reference_iterations_per_s"] for l in levels) else None,
           "budget_s": budget_s, "wall_s": time.perf_counter() - t_start,
           "protocol": "per level: 100 iterations / measured iterations per s (ours: device optimizer, graph-"
                       "replayed; reference: one getValueAndDerivative); parity at alpha = 0 on the same level"}
    if out["reference_s_per_pair_estimate"]:
        out["speedup_estimate"] = out["reference_s_per_pair_estimate"] / ours_total
    return out


def batch_compare(torch, steps=10, warmup=3, pairs=64):
    """Config 4: 64 config-2-style pairs of uneven sizes (64^3 .. 160x160x128), NCC/MSE mixed, all
    registered together, one persistent kernel per optimizer iteration (graph-replayed); aggregate
    voxel-evaluations per second = (sum of the pairs' voxels) x iterations / device time.  The
    intermediates (GBs) exceed the L2, so no flush is needed between iterations."""
    from skmimageregistration_b200 import workloads
    from skmimageregistration_b200.evaluator import Batch
    t0 = time.perf_counter()
    problems, metrics, odesc, info = workloads.make_batch(pairs, seed=0)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    b = Batch(problems, metrics, odesc)
    create_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.enqueue(0))
    b.evaluate()
    initial = [b.result(i)[0]["value"] for i in range(len(problems))]
    b.run(warmup)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    b.enqueue(steps)
    e.record(stream)
    torch.cuda.synchronize()
    b.run(0)                                            # raises if a bounded barrier gave up
    ms = s.elapsed_time(e) / steps
    voxels = info["total_voxels"]
    d = b.describe()
    states = [b.state(i) for i in range(len(problems))]
    out = {"config": info, "iterations_timed": steps, "ms_per_iteration": ms,
           "voxel_evaluations_per_s": voxels / (ms * 1e-3), "batch_iterations_per_s": 1e3 / ms,
           "kernel_launches_per_iteration": 1, "launch": d, "setup_s": {"generate": gen_s, "create_and_tune": create_s},
           "pairs_with_lower_value": int(sum(1 for st, v0 in zip(states, initial) if st["best_value"] < v0)),
           "timing": "CUDA events on the batch stream around graph-replayed iterations"}
    b.close()
    return out


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    from skmimageregistration_b200 import workloads
    from oracle import oracle as O
    pb, m, o, info = workloads.make(args.workload, seed=0, coefficients=O.bspline_coefficients)
    # each step is one full-size FP64 evaluation + update; bounded to ~2 minutes in total
    warm = min(args.warmup, 1)
    if warm:
        cpu_port_rate(pb, m, budget_s=0.0, max_steps=warm)
    rate, steps, el, threads = cpu_port_rate(pb, m, budget_s=90.0, max_steps=max(1, min(args.steps, 40)),
                                             min_steps=1)
    line = {
        "metric": "optimizer_iterations_per_s", "value": rate, "unit": "iter/s", "impl": "reference",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1e3 / rate,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(info, timing="CPU wall clock per full-size evaluation + update"),
        "cpu_baseline": {"value": rate, "unit": "iter/s", "cores": threads, "kind": "port",
                         "sample": "%d full-size 128x128x96 NCC+RD evaluations (FP64 restatement, OpenMP)" % steps},
        "e2e": {"value": rate, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        import torch
        if torch.cuda.is_available():
            r = reference_cuda_rate(pb, m)
            if r is not None:
                line["reference_cuda_evaluator"] = {
                    "value": r[0], "unit": "iter/s", "steps": r[1],
                    "note": "reference GpuKernelEvaluator (double build, -use_fast_math, sm_100a) driven like "
                            "its ITK glue; host loop, wall clock"}
    except Exception as exc:                                 # reported, not fatal
        line["reference_cuda_evaluator"] = {"unavailable": str(exc)[:200]}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from skmimageregistration_b200 import workloads
    from skmimageregistration_b200.evaluator import GpuKernelEvaluator, Optimizer

    torch.cuda.set_device(local_rank)
    pb, mdesc, odesc, info_cfg = workloads.make(args.workload, seed=rank)
    P = pb.num_parameters
    cpw = np.ones(pb.C)
    ev = GpuKernelEvaluator(pb)
    gemm_request = GpuKernelEvaluator.AUTO if args.gemm == "auto" else GpuKernelEvaluator.REQ_TABLE_CUDA_CORES
    ev.path(gemm_request)
    opt = Optimizer(ev, odesc, mdesc, np.zeros(P), cpw)
    stream = torch.cuda.ExternalStream(opt.enqueue(0))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # warm-up
    opt.enqueue(args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.25)
    with torch.cuda.stream(stream):
        for i in range(args.steps):
            flush.fill_(float(i))                   # evict L2 (256 MB > 126 MB) outside the events
            starts[i].record(stream)
            opt.enqueue(1)
            ends[i].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = sum(s.elapsed_time(e) for s, e in zip(starts, ends))
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * args.steps / (ms * 1e-3)
    kernels_per_iter = opt.graph_kernel_count()

    # per-phase timing (CUDA events on the evaluator's stream, same iteration un-graphed)
    prof_iters = min(max(args.steps, 20), 200)
    phases = opt.profile(prof_iters)
    state = opt.state()

    # e2e: reference-facing C-ABI call with host buffers + host-side optimizer update
    e2e_steps = args.e2e_steps or min(args.steps, 300)
    ev2 = GpuKernelEvaluator(pb)
    ev2.path(gemm_request)
    # the caller's parameter and derivative arrays in page-locked host memory: the metric call's
    # kernels read the parameters and write the derivative across the bus, with no staging copies
    def pinned(n):
        return torch.zeros(n, dtype=torch.float64, pin_memory=True).numpy()
    from scipy.linalg.blas import daxpy, ddot
    params = pinned(P)
    grad = [pinned(P), pinned(P)]                    # this and the previous step's derivative
    t_sim = 0.0
    ev2.metric(mdesc, params, cpw)                  # warm-up
    ddot(grad[0], grad[1])
    daxpy(grad[0], params, a=0.0)
    # three chunks of steps, the median chunk's rate reported (a host hiccup in one chunk does not
    # move it); every step: L2 flush and synchronise outside the clock, then the metric call and the
    # host update inside it
    chunk_rates, e2e_s = [], 0.0
    nchunk = max(1, e2e_steps // 3)
    for c0 in range(0, e2e_steps, nchunk):
        c_s = 0.0
        for i in range(c0, min(e2e_steps, c0 + nchunk)):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g, prev = grad[i & 1], grad[(i + 1) & 1]
            v, _ = ev2.metric(mdesc, params, cpw, out_derivative=g)
            # AdaptiveStepGradientDescentOptimizerv4 update on the host (ITK glue path), in place
            # with BLAS: the step base is the previous position, so params += lr * g
            lr = odesc.a / (odesc.A + t_sim + 1.0) ** odesc.alpha
            sp = ddot(g, prev)
            daxpy(g, params, a=lr)
            x = -sp
            t_sim = max(0.0, t_sim + odesc.f_min + (odesc.f_max - odesc.f_min) /
                        (1.0 - (odesc.f_max / odesc.f_min) * math.exp(-x / odesc.omega)))
            c_s += time.perf_counter() - t0
        chunk_rates.append((min(e2e_steps, c0 + nchunk) - c0) / c_s)
        e2e_s += c_s
    e2e_rate = sorted(chunk_rates)[len(chunk_rates) // 2]
    if world > 1:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_rate = world * e2e_steps / float(t.item())
    h2d = P * 8                                     # parameters; identical weights are not sent again
    d2h = P * 8 + 10 * 8

    line = None
    if rank == 0:
        hbm_peak, hbm_src = measured_peaks()
        fp32_peak = fp32_peak_tflops(torch)
        tf32_peak = tf32_peak_tflops(torch)
        info = ev.describe()
        # the phases are timed un-graphed with events between them; scale them to the graphed
        # iteration that `value` measures, so that per-kernel and per-step figures describe one run
        phase_sum = sum(v for k, v in phases.items() if k != "update")
        scale = (ms / args.steps) / phase_sum if phase_sum > 0 else 1.0
        phases_graph = {k: v * scale for k, v in phases.items()}
        kernels = kernel_work(pb, info, phases_graph)
        for k, v in kernels.items():
            v["ms_ungraphed"] = v["ms"] / scale
        dom = max(kernels, key=lambda k: kernels[k]["ms"])
        kd = kernels[dom]
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "traffic_%s.json" % args.workload)
        if os.path.exists(tpath):
            try:
                traffic = json.load(open(tpath)).get(kd["name"])
            except Exception:
                traffic = None
        for k, v in kernels.items():
            v["tflops"] = v["flops"] / (v["ms"] * 1e-3) / 1e12 if v["ms"] > 0 else None
            v["gbs"] = v["bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] > 0 else None
            v["fp32_frac"] = v["tflops"] / fp32_peak if v["tflops"] is not None else None
            v["hbm_frac"] = v["gbs"] / hbm_peak if v["gbs"] is not None else None
            v["alg_gbs"] = v["alg_bytes"] / (v["ms"] * 1e-3) / 1e9 if v["ms"] > 0 else None
            v["alg_hbm_frac"] = v["alg_gbs"] / hbm_peak if v["alg_gbs"] is not None else None
            if "tensor_flops" in v:
                v["tensor_tflops"] = v["tensor_flops"] / (v["ms"] * 1e-3) / 1e12 if v["ms"] > 0 else None
                v["tensor_frac"] = v["tensor_tflops"] / tf32_peak if v["tensor_tflops"] is not None else None
        if kd["bound"] == "tensor":
            roof = {"kernel": kd["name"], "bound": "tensor", "achieved": kd["tensor_tflops"], "peak": tf32_peak,
                    "unit": "TFLOP/s", "frac": kd["tensor_frac"], "traffic": traffic,
                    "peak_source": "cuBLAS FP32 GEMM 8192^3 with TF32 tensor cores, measured live in this run",
                    "tensor_flops_per_launch": kd["tensor_flops"], "fp32_equivalent_tflops": kd["tflops"],
                    "flops_per_launch": kd["flops"], "launch_ms": kd["ms"],
                    "hbm": {"achieved": kd["gbs"], "peak": hbm_peak, "unit": "GB/s", "frac": kd["hbm_frac"],
                            "algorithmic_bytes_per_launch": kd["bytes"], "peak_source": hbm_src}}
        elif kd["bound"] == "fp32":
            roof = {"kernel": kd["name"], "bound": "fp32", "achieved": kd["tflops"], "peak": fp32_peak,
                    "unit": "TFLOP/s", "frac": kd["fp32_frac"], "traffic": traffic,
                    "peak_source": "cuBLAS SGEMM 8192^3, TF32 off, measured live in this run (CUDA-core FP32)",
                    "flops_per_launch": kd["flops"], "launch_ms": kd["ms"],
                    "hbm": {"achieved": kd["gbs"], "peak": hbm_peak, "unit": "GB/s", "frac": kd["hbm_frac"],
                            "algorithmic_bytes_per_launch": kd["bytes"], "peak_source": hbm_src}}
        else:
            roof = {"kernel": kd["name"], "bound": "hbm", "achieved": kd["alg_gbs"], "peak": hbm_peak, "unit": "GB/s",
                    "frac": kd["alg_hbm_frac"], "traffic": traffic, "peak_source": hbm_src,
                    "algorithmic_bytes_per_launch": kd["alg_bytes"], "launch_ms": kd["ms"],
                    "basis": "fused: 8 B per fixed voxel (fixed value + moving coefficient)",
                    "design_bytes_per_launch": kd["bytes"], "design_gbs": kd["gbs"], "design_frac": kd["hbm_frac"]}
        line = {
            "metric": "optimizer_iterations_per_s", "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded %s pair per GPU)" % args.workload,
            "config": dict(info_cfg, parallelism="pair-parallel x%d (independent replicas, no collective)" % world,
                           kernel_path={1: "generic", 2: "phase table (CUDA-core GEMMs)",
                                        3: "phase table (tcgen05 3xTF32 GEMMs)"}[info["path"]],
                           l2="flushed before every timed iteration (256 MB write outside the events)",
                           timing="CUDA events on the evaluator stream around each graph-replayed iteration",
                           arithmetic="FP32 kernel sums, FP64 global sums"),
            "clocks": clocks,
            "gpu_launches": kernels_per_iter * args.steps,
            "kernels_per_iteration": kernels_per_iter,
            "phases_ms": phases,
            "final_state": state,
            "roofline": roof,
            "roofline_iteration": iteration_roofline(pb, ms / args.steps, hbm_peak, hbm_src, fp32_peak),
            "roofline_kernels": kernels,
            "phase_scale_to_graph": scale,
            "peaks": {"hbm_gbs": hbm_peak, "hbm_source": hbm_src, "fp32_sgemm_tflops": fp32_peak,
                      "tf32_gemm_tflops": tf32_peak},
            "e2e": {"value": e2e_rate, "unit": "iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "chunk_rates": [round(r, 1) for r in chunk_rates],
                    "host_update": "BLAS ddot + daxpy on the page-locked arrays"},
        }
    opt.close()
    ev.close()
    ev2.close()
    if rank == 0 and world == 1 and not args.no_multiscale:
        line["multiscale"] = multiscale_compare("ncc128")
        line["multiscale_mse2d"] = multiscale_compare("mse2d")
        # with L1 1e-3 every MSE gradient component stays below the L1 threshold, so the plain method
        # (ours and the reference alike) keeps alpha = 0; a weaker L1 shows the registration moving
        line["multiscale_mse2d_l1_1e-6"] = multiscale_compare("mse2d", dict(reg_l1=[1e-6]))
    if rank == 0 and world == 1 and not args.no_batch:
        line["batch64"] = batch_compare(torch)
    if rank == 0 and world == 1 and not args.no_ct3d:
        line["ct3d"] = ct3d_compare(torch)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O  # noqa: F401  (CPU baseline leg only)
        rate, steps, el, threads = cpu_port_rate(pb, mdesc, budget_s=15.0, max_steps=5)
        line["cpu_baseline"] = {"value": rate, "unit": "iter/s", "cores": threads, "kind": "port",
                                "sample": "%d full-size evaluations + update, FP64 restatement, %.1f s" % (steps, el)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def spawn_ranks(n):
    """`bench.py --gpus N` started without a launcher: re-run this script under torchrun with one
    process per GPU (127.0.0.1 rendezvous, a free port), bounded by an outer timeout."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", str(n), "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.only != "all":                          # one secondary line alone (profiling, quick checks)
        import torch
        if args.only == "batch":
            out = batch_compare(torch, steps=args.steps, warmup=args.warmup, pairs=args.batch_pairs)
        elif args.only == "ct3d":
            out = ct3d_compare(torch)
        else:
            out = multiscale_compare(args.only)
        print(json.dumps(out), flush=True)
        return 0
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        return run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
