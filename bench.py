"""Benchmark: fitted texels/s of the SVBRDF fit (81x81 directions) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one step): the svbrdffit texel loop over a 400x400-texel synthetic
BTF with the 81-direction ring layout (6561 direction pairs), RGB FP32 samples,
the uneven parameter mix (20% near-diffuse, 10% strongly anisotropic) -- the
batched persistent fit of 400x400 texels.  Per texel: luminance slice, the
reference's default initial guess (NDF -> PCA -> SGGX projection), LM
(max 1024 iterations, Fresnel 1) and the five output maps.

* value: texels/s with the samples resident in HBM (12.6 GB, larger than L2),
  timed with CUDA events on the library's stream, max over ranks.
* e2e: the same through the public C ABI with pinned HOST buffers: the step's
  samples are copied host->device and all maps device->host inside the timed
  region.
* roofline: the LM kernel (the dominant kernel) against the FP32 CUDA-core peak
  (SMs x 128 lanes x 2 flops x SM clock sampled under load), with its
  algorithmic flops counted per ordered direction pair (169 per Jacobian
  evaluation, 33 per residual, an FMA counted as 2);
  traffic per texel from an ncu capture of a 160x160-texel case.
* roofline_ndf: the NDF GEMM of the default initial guess (tcgen05 tensor
  cores) against the measured BF16 peak in MEASURED_PEAKS.json.
* cpu_baseline: the reference's own CPU fitter (oracle/_ref, compiled from the
  reference's sources) on a bounded sample of the same texels, all host cores.

Multi-GPU: texels are independent; each rank fits its own 400x400 shard (weak
scaling), no data-path collective.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "fitted texels/s (81x81 dirs) at residual <=1.01x plain LM; % of FP32/HBM peak"
SEED, MIX = 2024, 1
WIDTH = HEIGHT = 400
# Algorithmic flops of an analytic-Jacobian LM per ordered direction pair (FMA = 2),
# counted from svf_model.cuh::eval_pair plus the packed J^T J / J^T r accumulation:
# a Jacobian evaluation (accepted steps and the start point) and a residual
# evaluation (every trial).  The kernel evaluates the specular core once per
# unordered pair (svf_lm.cu::sym_pair), so it executes fewer.
FLOPS_JACOBIAN_PASS = 169
FLOPS_RESIDUAL_PASS = 33
# DRAM bytes per texel of lm_fit_kernel, measured by ncu on a 160x160-texel ring-81
# capture (dram__bytes_read.sum + dram__bytes_write.sum = 675.3 MB + 6.6 MB for
# 25600 texels; the luminance slab is read once).
LM_DRAM_BYTES_PER_TEXEL = (675.3e6 + 6.6e6) / 25600
# DRAM bytes per texel of ndf_tc_kernel over the operator's non-empty tiles,
# measured by ncu on the same case (1.95 GB + 332 MB for 25600 texels).
NDF_DRAM_BYTES_PER_TEXEL = (1.95e9 + 332e6) / 25600
NDF_ROWS, NDF_ROWS_PAD = 3217, 3328   # 64x64 NDF texels inside the hemisphere, padded to the tile


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 10 ms on a thread (read-only queries), and
    nvidia-smi at 200 ms, whose samples are reported where NVML gave none."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown", 0x8),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap", 0x4))

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", f"svf_clocks_{os.getpid()}.csv")
        self.nvml = None
        self.rows = []
        self.smi_id = str(device_index)
        try:   # the same physical GPU as the CUDA ordinal, whatever CUDA_VISIBLE_DEVICES says
            import torch

            self.smi_id = "GPU-" + str(torch.cuda.get_device_properties(device_index).uuid)
        except Exception:
            pass
        try:
            import pynvml

            pynvml.nvmlInit()
            try:
                handle = pynvml.nvmlDeviceGetHandleByUUID(self.smi_id)
            except Exception:
                handle = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.nvml = (pynvml, handle)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None

    def _poll(self):
        pynvml, h = self.nvml
        while not self.stop_evt.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                try:
                    bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                except Exception:
                    bits = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.rows.append((float(sm), int(bits)))
            except Exception:
                pass
            self.stop_evt.wait(0.01)

    def __enter__(self):
        if self.nvml:
            import threading

            self.stop_evt = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
        # nvidia-smi alongside: its samples stand in if NVML delivered none
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.smi_id}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.nvml:
            self.stop_evt.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.nvml and self.rows:
            pynvml = self.nvml[0]
            reasons = set()
            for _, bits in self.rows:
                for name, const, default in self.REASONS:
                    if bits & getattr(pynvml, const, default):
                        reasons.add(name)
            sm = np.array([r[0] for r in self.rows])
            return {"sm_mhz": float(np.median(sm)), "sm_mhz_min": float(sm.min()), "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(reasons), "samples": len(self.rows), "source": "nvml, 10 ms"}
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = np.array([float(r[1]) for r in rows])
        reasons = set()
        for r in rows:
            for name, val in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                                 r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def ring81_mesh():
    import tempestrenderer_b200 as svf

    lp = svf.directions_ring81()
    tri, edges, angles = svf.triangulate(lp)
    return svf.Layout(lp, tri, edges, angles)


# ----------------------------------------------------------------------------
# the reference's CPU fitter
# ----------------------------------------------------------------------------

def reference_fit_rate(texels: int, first: int = 0, threads: int | None = None, indices=None):
    """Times the reference's texel loop (oracle/_ref) on `texels` texels of the
    benchmark BTF (texels first.. or the given texel indices), all host threads;
    returns (texels/s, seconds, threads, per-texel RMSE)."""
    import oracle

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libtempest_ref.so is not built")
    threads = threads or os.cpu_count() or 1
    tp = oracle.ring81_angles()
    lp = oracle.angles_to_parabolic(tp)
    idx = list(range(first, first + texels)) if indices is None else [int(i) for i in indices]
    rgb = np.stack([oracle.synth_render(SEED, t, oracle.synth_truth(SEED, MIX, t), lp) for t in idx])
    btf = oracle.RefBTF.from_texels(tp, rgb)
    secs, rmse = btf.time_fit(0, len(idx), threads, 0)
    return len(idx) / secs, secs, threads, np.asarray(rmse, np.float64)


# Texels of the benchmark BTF that the reference also fits for the parity block:
# PARITY_TEXELS indices spread evenly over the 400x400 texels.
PARITY_TEXELS = 256


def parity_indices(T: int, n: int = PARITY_TEXELS):
    return np.unique(np.linspace(0, T - 1, n).round().astype(np.int64))


def parity_block(gpu_rmse, ref_rmse):
    """Per-texel final RMSE of the GPU fit over the reference CPU fit's, same texels."""
    g, r = np.asarray(gpu_rmse, np.float64), np.asarray(ref_rmse, np.float64)
    ratio = g / np.maximum(r, 1e-30)
    # (the reference's LM ends some texels far above the GPU fit -- a few percent with
    # an RMSE several times the GPU's -- so the ratio of mean RMSEs sits far below the
    # per-texel median; both are reported)
    return {"texels": int(len(g)), "mean_rmse_ratio": float(g.mean() / r.mean()),
            "mean_of_texel_ratios": float(ratio.mean()), "median_ratio": float(np.median(ratio)),
            "within_1pct": float(np.mean(ratio <= 1.01)), "p99_ratio": float(np.quantile(ratio, 0.99)),
            "max_ratio": float(ratio.max()), "below_0.99": float(np.mean(ratio < 0.99)),
            "below_0.5": float(np.mean(ratio < 0.5)), "gpu_mean_rmse": float(g.mean()), "reference_mean_rmse": float(r.mean())}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    sample = max(16, 2 * threads)
    for _ in range(args.warmup):
        reference_fit_rate(min(sample, 16), threads=threads)
    rates, secs_total, done = [], 0.0, 0
    for k in range(args.steps):
        rate, secs, thr, _ = reference_fit_rate(sample, first=k * sample, threads=threads)
        rates.append(rate)
        secs_total += secs
        done += sample
    value = done / secs_total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "texels/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
            "data": "synthetic",
            "config": {"workload": f"svbrdffit texel loop, {WIDTH}x{HEIGHT} texels, ring-81 layout, RGB FP32, "
                                   f"mix 20% near-diffuse/10% anisotropic, default init, LM 1024 max",
                       "texels_per_step": sample, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "texels/s", "cores": threads, "kind": "reference",
                             "sample": f"{sample} texels of the benchmark BTF per step, {threads} worker threads"},
            "e2e": {"value": value, "unit": "texels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# the GPU fitter
# ----------------------------------------------------------------------------

def _normal_of_quat(q):
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    n = np.stack([2 * (x * z + y * w), 2 * (y * z - x * w), 1 - 2 * (x * x + y * y)], 1)
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def _quat_of_euler(e):
    h = 0.5 * e.astype(np.float64)
    s1, c1, s2, c2, s3, c3 = np.sin(h[:, 0]), np.cos(h[:, 0]), np.sin(h[:, 1]), np.cos(h[:, 1]), np.sin(h[:, 2]), \
        np.cos(h[:, 2])
    return np.stack([s1 * c2 * c3 + c1 * s2 * s3, -s1 * c2 * s3 + c1 * s2 * c3, c1 * c2 * s3 + s1 * s2 * c3,
                     c1 * c2 * c3 - s1 * s2 * s3], 1)


def param_error(params, truth):
    """Fitted 7-parameter luminance model against the synthetic ground truth
    ([T][16]: kd rgb, ks rgb, sigma, quaternion, euler, kind): normal angle, the
    lobe's geometric-mean scale and anisotropy, the luminance albedos."""
    p, t = np.asarray(params, np.float64), np.asarray(truth, np.float64)
    w = np.array([0.2126, 0.7152, 0.0722])
    ang = np.degrees(np.arccos(np.clip(np.abs((_normal_of_quat(_quat_of_euler(p[:, 4:7])) *
                                               _normal_of_quat(t[:, 8:12])).sum(1)), 0, 1)))
    gm = np.abs(np.log(np.sqrt(np.abs(p[:, 0] * p[:, 1]) + 1e-12) / np.sqrt(t[:, 6] * t[:, 7])))
    an = lambda a, b: np.log(np.maximum(a, b) / np.maximum(np.minimum(a, b), 1e-6))
    aniso = np.abs(an(np.abs(p[:, 0]), np.abs(p[:, 1])) - an(t[:, 6], t[:, 7]))
    kd, ks = t[:, 0:3] @ w, t[:, 3:6] @ w
    ekd = np.abs(p[:, 3] - kd) / np.maximum(kd, 0.02)
    eks = np.abs(p[:, 2] - ks) / np.maximum(ks, 0.02)
    q = lambda a: {"median": float(np.median(a)), "p90": float(np.quantile(a, 0.9))}
    return {"normal_deg": q(ang), "log_scale": q(gm), "log_anisotropy": q(aniso), "kd_rel": q(ekd), "ks_rel": q(eks)}


def config3_item(svf, ctx, layout, model, steps, dev, side=1024):
    """1024x1024 texels, ring-81, FP16 samples: the plain GPU LM (default guess)
    against the learned guess + LM, with their residuals and ground-truth errors."""
    import torch

    T = side * side
    N = layout.light_count ** 2
    samples = torch.empty((T, N, 3), dtype=torch.float16, device=dev)
    truth = torch.empty((T, 16), dtype=torch.float32, device=dev)
    ctx.synth_btf(SEED + 3, MIX, layout.lights_parabolic, 0, T, samples, sample_type=svf.SVF_SAMPLES_F16,
                  truth=truth)
    opts = svf.options(max_iterations=1024)
    res = {}
    for name, mlp in (("plain", None), ("learned", model)):
        maps = {k: torch.zeros(s_, dtype=torch.float32, device=dev) for k, s_ in
                {"rmse": (T,), "params": (T, 7)}.items()}
        run = lambda: ctx.fit_texels(layout, samples, side, side, sample_type=svf.SVF_SAMPLES_F16, opts=opts,
                                     want=tuple(maps), out=maps, check=False, mlp=mlp)[1]
        run()
        st = [run() for _ in range(steps)]
        ms = sum(r.ms_total for r in st) / steps
        res[name] = (ms, maps["rmse"].cpu().numpy(), maps["params"].cpu().numpy(), st[-1])
    truth_np = truth.cpu().numpy()
    del samples, truth
    torch.cuda.empty_cache()
    (pms, prm, ppar, prs), (lms, lrm, lpar, lrs) = res["plain"], res["learned"]
    ratio = lrm / np.maximum(prm, 1e-12)
    return {"workload": f"{side}x{side} texels, ring-81, FP16 RGB in HBM ({T * N * 6 / 1e9:.1f} GB), mix 20% "
                        f"near-diffuse/10% anisotropic",
            "plain": {"value": T / (pms / 1e3), "unit": "texels/s", "ms": pms, "mean_rmse": float(prm.mean()),
                      "mean_iterations": prs.iterations / T, "ground_truth_error": param_error(ppar, truth_np)},
            "learned": {"value": T / (lms / 1e3), "unit": "texels/s", "ms": lms, "mean_rmse": float(lrm.mean()),
                        "mean_iterations": lrs.iterations / T, "ground_truth_error": param_error(lpar, truth_np),
                        "failed_texels": int(lrs.failed_texels)},
            "speedup": pms / lms,
            "residual_ratio": {"mean": float(lrm.mean() / prm.mean()), "median": float(np.median(ratio)),
                               "within_1pct": float(np.mean(ratio <= 1.01)),
                               # the reference's LM stops at MSE <= 1e-6 (fitting.hh:557): a texel whose RMSE
                               # is at or below 1e-3 has met its own target whatever the other fit reached
                               "within_1pct_or_at_target": float(np.mean((ratio <= 1.01) | (lrm <= 1e-3))),
                               "learned_at_target": float(np.mean(lrm <= 1e-3)),
                               "plain_at_target": float(np.mean(prm <= 1e-3))}}


def learned_init_item(svf, ctx, layout, samples, W, H, ref_rmse, steps, dev, truth=None):
    """The learned initial guess (SVF_INIT_MLP) on the benchmark texels: train a model on
    separately seeded synthetic texels, then fit the same texels from its prediction."""
    import torch

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    topts = svf.mlp_train_options()   # the defaults: 2^20 texels, 48 epochs
    model, loss = svf.Mlp.train(ctx, layout.lights_parabolic, topts)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    T = W * H
    maps = {k: torch.zeros(s, dtype=torch.float32, device=dev) for k, s in
            {"rmse": (T,), "params": (T, 7)}.items()}
    opts = svf.options(max_iterations=1024)
    run = lambda: ctx.fit_texels(layout, samples, W, H, opts=opts, want=tuple(maps), out=maps, check=False,
                                 mlp=model)[1]
    run()
    st = [run() for _ in range(steps)]
    ms = sum(r.ms_total for r in st) / steps
    rmse = maps["rmse"].cpu().numpy()
    ratio = rmse / np.maximum(ref_rmse, 1e-12)
    # the plain-LM fallback at the median relative residual: about half the texels
    # are fitted from the default guess as well and keep the lower RMSE
    lum_rms = torch.sqrt(((0.2126 * samples[..., 0] + 0.7152 * samples[..., 1] + 0.0722 * samples[..., 2])
                          .double() ** 2).mean(1)).cpu().numpy()
    th = float(np.median(rmse / lum_rms))
    fmaps = {k: torch.zeros_like(v) for k, v in maps.items()}
    frun = lambda: ctx.fit_texels(layout, samples, W, H, opts=opts, want=tuple(fmaps), out=fmaps, check=False,
                                  mlp=model, fallback=th)[1]
    frun()
    fst = [frun() for _ in range(steps)]
    fms = sum(r.ms_total for r in fst) / steps
    frmse = fmaps["rmse"].cpu().numpy()
    fratio = frmse / np.maximum(ref_rmse, 1e-12)
    del fmaps
    cfg3 = config3_item(svf, ctx, layout, model, steps, dev)
    model.close()
    return {"value": T / (ms / 1e3), "unit": "texels/s", "ms_per_step": ms, "steps": steps,
            "phases_ms": {"luminance": sum(r.ms_luminance for r in st) / steps,
                          "init": sum(r.ms_init for r in st) / steps, "lm": sum(r.ms_fit for r in st) / steps},
            "lm_work": {"jacobian_passes": st[-1].jacobians, "residual_passes": st[-1].residuals,
                        "failed_texels": st[-1].failed_texels, "mean_iterations": st[-1].iterations / T},
            "mean_rmse": float(rmse.mean()), "default_init_mean_rmse": float(ref_rmse.mean()),
            "ground_truth_error": None if truth is None else param_error(maps["params"].cpu().numpy(), truth),
            "rmse_ratio_vs_default_init": {"median": float(np.median(ratio)), "within_1pct": float(np.mean(ratio <= 1.01)),
                                           "better_1pct": float(np.mean(ratio < 0.99)), "p90": float(np.quantile(ratio, 0.9))},
            "training": {"seconds": train_s, "final_loss": loss, "texels": topts.texels, "epochs": topts.epochs,
                         "lr": topts.lr},
            "config3_1024x1024_fp16": cfg3,
            "with_fallback": {"value": T / (fms / 1e3), "unit": "texels/s", "ms_per_step": fms,
                              "threshold_relative_rmse": th, "fallback_texels": fst[-1].fallback_texels,
                              "mean_rmse": float(frmse.mean()),
                              "rmse_ratio_vs_default_init": {"median": float(np.median(fratio)),
                                                             "within_1pct": float(np.mean(fratio <= 1.01)),
                                                             "p90": float(np.quantile(fratio, 0.9))}},
            "model": "MLP 96-256-256-8 (64 half-vector bins + 32 pairs of the luminance slab -> log S, ks, kd), "
                     "features from the luminance pass, hidden layers on the tcgen05 tensor cores (BF16x3, FP32 "
                     "accuracy); LM from its prediction with 1e-4 of the reference's initial damping (the library default for the learned guess)"}


def _fp64_brdf_rows(args):
    """The FP64 oracle's BRDF (svfo_brdf_f64) of 7-parameter vectors over all pairs
    of a layout: rows as FP32 and each row's RMS in FP64 (a worker of a spawned pool)."""
    import oracle

    params, lp = args
    rows = np.zeros((len(params), lp.shape[0] ** 2), np.float32)
    rms = np.zeros(len(params))
    ref32 = np.zeros(len(params))
    for i, p in enumerate(params):
        f32, f64 = oracle.brdf_all(np.asarray(p, np.float64), lp)
        rows[i] = f64
        rms[i] = np.sqrt(np.mean(f64 ** 2))
        # the reference's own FP32 evaluation (the oracle restates it bit for bit)
        ref32[i] = np.sqrt(np.mean((f32.astype(np.float64) - f64) ** 2)) / max(rms[i], 1e-30)
    return rows, rms, ref32


def fp64_check(svf, ctx, lp, params, chunk=512):
    """BRDF relative error of the GPU's FP32 model against the FP64 oracle at the
    given parameters: per texel RMS(GPU - FP64) / RMS(FP64) over all pairs, read as
    the RMSE of a zero-iteration GPU fit to the FP64 values."""
    import multiprocessing as mp

    n = len(params)
    parts = [(params[i:i + chunk], lp) for i in range(0, n, chunk)]
    err = np.zeros(n)
    with mp.get_context("spawn").Pool(min(len(parts) * 4, os.cpu_count() or 1)) as pool:
        sub = [(p[j:j + 32], lp) for p, _ in parts for j in range(0, len(p), 32)]
        res = pool.map(_fp64_brdf_rows, sub)
    rows = np.concatenate([r[0] for r in res])
    rms = np.concatenate([r[1] for r in res])
    ref32 = np.concatenate([r[2] for r in res])
    for i in range(0, n, chunk):
        _, rmse, _ = ctx.lsq_fit_batch(lp, rows[i:i + chunk], np.ascontiguousarray(params[i:i + chunk], np.float32),
                                       svf.options(max_iterations=0))
        err[i:i + chunk] = rmse / np.maximum(rms[i:i + chunk], 1e-30)
    return err, ref32


def fib151_item(svf, ctx, steps, dev, side=768):
    """768x768 texels on the 151-direction Fibonacci layout (22801 pairs), FP16 RGB samples;
    BRDF error against the FP64 oracle and parameter error against the ground truth on a
    seeded 4096-texel subset."""
    import torch

    lp = svf.directions_fibonacci(151)
    layout = svf.Layout(lp, *svf.triangulate(lp))
    N = 151 * 151
    T = side * side
    samples = torch.empty((T, N, 3), dtype=torch.float16, device=dev)
    truth = torch.empty((T, 16), dtype=torch.float32, device=dev)
    ctx.synth_btf(SEED + 2, MIX, lp, 0, T, samples, sample_type=svf.SVF_SAMPLES_F16, truth=truth)
    maps = {k: torch.zeros(s, dtype=torch.float32, device=dev) for k, s in
            {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
             "params": (T, 7)}.items()}
    opts = svf.options(max_iterations=1024)
    run = lambda: ctx.fit_texels(layout, samples, side, side, sample_type=svf.SVF_SAMPLES_F16, opts=opts,
                                 want=tuple(maps), out=maps, check=False)[1]
    run()
    st = [run() for _ in range(steps)]
    ms = sum(r.ms_total for r in st) / steps
    ms_fit = sum(r.ms_fit for r in st) / steps
    flops = N * (FLOPS_JACOBIAN_PASS * st[-1].jacobians + FLOPS_RESIDUAL_PASS * st[-1].residuals)
    out = {"value": T / (ms / 1e3), "unit": "texels/s", "ms_per_step": ms, "steps": steps,
           "workload": f"{side}x{side} texels, Fibonacci-151 layout (22801 pairs), FP16 RGB in HBM "
                       f"({samples.numel() * 2 / 1e9:.1f} GB), mix 20% near-diffuse/10% anisotropic, default init",
           "phases_ms": {"luminance": sum(r.ms_luminance for r in st) / steps,
                         "init": sum(r.ms_init for r in st) / steps,
                         "ndf_gemm": sum(r.ms_ndf for r in st) / steps, "lm": ms_fit},
           "lm_tflops": flops / (ms_fit / 1e3) / 1e12,
           "failed_texels": st[-1].failed_texels, "mean_rmse": float(maps["rmse"].mean().item())}
    params = maps["params"].cpu().numpy()
    truth_np = truth.cpu().numpy()
    del samples, truth
    torch.cuda.empty_cache()
    idx = np.sort(np.random.default_rng(SEED + 2).choice(T, 4096, replace=False))
    err, ref32 = fp64_check(svf, ctx, lp, params[idx])
    q = lambda a: {"median": float(np.median(a)), "p99": float(np.quantile(a, 0.99)), "max": float(a.max())}
    out["fp64_check"] = {"texels": len(idx), "subset": "4096 texels drawn with seed SEED + 2",
                         "brdf_rel_error": q(err), "bar": 1e-5, "within_bar": float(np.mean(err <= 1e-5)),
                         "reference_fp32_brdf_rel_error": dict(q(ref32), within_bar=float(np.mean(ref32 <= 1e-5))),
                         "ground_truth_error_subset": param_error(params[idx], truth_np[idx]),
                         "ground_truth_error_all": param_error(params, truth_np)}
    out["fp64_check_summary"] = {"brdf_rel_error_max": float(err.max()), "within_1e-5": float(np.mean(err <= 1e-5)),
                                 "reference_fp32_within_1e-5": float(np.mean(ref32 <= 1e-5)),
                                 "normal_p90_deg": out["fp64_check"]["ground_truth_error_subset"]["normal_deg"]["p90"]}
    return out


def batch_item(svf, ctx, steps, dev):
    """Eight BTFs of uneven sizes and two layouts in one svf_fit_btfs call (FP16 RGB)."""
    import torch

    ring = ring81_mesh()
    lp151 = svf.directions_fibonacci(151)
    fib = svf.Layout(lp151, *svf.triangulate(lp151))
    shapes = [(ring, 128), (ring, 256), (ring, 512), (ring, 1024), (fib, 128), (fib, 256), (fib, 384), (fib, 512)]
    btfs = []
    for i, (lay, side) in enumerate(shapes):
        L = lay.light_count
        s = torch.empty((side * side, L * L, 3), dtype=torch.float16, device=dev)
        ctx.synth_btf(SEED + 10 + i, MIX, lay.lights_parabolic, 0, side * side, s, sample_type=svf.SVF_SAMPLES_F16)
        btfs.append(dict(layout=lay, samples=s, width=side, height=side, sample_type=svf.SVF_SAMPLES_F16))
    total_gb = sum(b["samples"].numel() * 2 for b in btfs) / 1e9
    opts = svf.options(max_iterations=1024)
    ctx.fit_btfs(btfs, opts=opts, want=("rmse",), check=False)
    for _ in range(steps):
        maps, runs, total = ctx.fit_btfs(btfs, opts=opts, want=("rmse", "stats"), check=False)
    T = sum(b["width"] * b["height"] for b in btfs)
    # each BTF alone (its own svf_fit_texels call): its texels/s
    alone = []
    for b in btfs:
        fit1 = lambda: ctx.fit_texels(b["layout"], b["samples"], b["width"], b["height"],
                                      sample_type=svf.SVF_SAMPLES_F16, opts=opts, want=("rmse",), check=False)[1]
        fit1()
        alone.append(fit1().ms_total)
    # the same batch from the learned guess: one model per layout (2^18 texels, 12 epochs)
    t0 = time.perf_counter()
    models = {id(lay): svf.Mlp.train(ctx, lay.lights_parabolic,
                                     svf.mlp_train_options(texels=1 << 18, epochs=12, batch=2048))[0]
              for lay in (ring, fib)}
    train_s = time.perf_counter() - t0
    lbtfs = [dict(b, mlp=models[id(b["layout"])]) for b in btfs]
    ctx.fit_btfs(lbtfs, opts=opts, want=("rmse",), check=False)
    lmaps, lruns, ltotal = ctx.fit_btfs(lbtfs, opts=opts, want=("rmse", "stats"), check=False)
    per = []
    for (lay, side), m, r, lm, ms1 in zip(shapes, maps, runs, lmaps, alone):
        it, lit = m["stats"]["iterations"], lm["stats"]["iterations"]
        ratio = lm["rmse"] / np.maximum(m["rmse"], 1e-12)
        per.append({"btf": f"{side}x{side} @ {lay.light_count}", "texels": int(r.texels),
                    "texels_per_s": side * side / (ms1 / 1e3), "ms_alone": ms1,
                    "iterations_p50": float(np.percentile(it, 50)), "iterations_p99": float(np.percentile(it, 99)),
                    "mean_rmse": float(m["rmse"].mean()), "max_rmse": float(m["rmse"].max()),
                    "failed_texels": int(r.failed_texels),
                    "learned": {"iterations_p50": float(np.percentile(lit, 50)),
                                "iterations_p99": float(np.percentile(lit, 99)),
                                "mean_rmse": float(lm["rmse"].mean()),
                                "residual_ratio_vs_plain": {"mean": float(lm["rmse"].mean() / m["rmse"].mean()),
                                                            "median": float(np.median(ratio)),
                                                            "max": float(ratio.max())}}})
    for mdl in models.values():
        mdl.close()
    for b in btfs:
        del b["samples"]
    torch.cuda.empty_cache()
    return {"value": T / (total.ms_total / 1e3), "unit": "texels/s", "ms_per_call": total.ms_total,
            "texels": T, "samples_gb": total_gb, "per_btf": per,
            "learned": {"value": T / (ltotal.ms_total / 1e3), "unit": "texels/s", "ms_per_call": ltotal.ms_total,
                        "training_s": train_s, "failed_texels": int(ltotal.failed_texels)},
            "note": "each BTF's maps equal its own svf_fit_texels fit bit for bit (tests/test_gpu_batch.py), "
                    "so the residual ratio to plain per-BTF LM is 1 by construction"}


def dfmf_bytes(theta_phi, width, height, u_planes, sxv_planes, data_size=2):
    """A DFMF file image (the layout LoadBTF parses, src/image/btf.cc:389-843): one
    (U [L*L][K], SxV [W*H][K]) plane pair per channel; SxV rows are file columns."""
    import struct

    dt = {2: np.float16, 4: np.float32}[data_size]
    tp = np.ascontiguousarray(theta_phi, np.float32)
    L = tp.shape[0]
    parts = [b"!DFMF08FC", struct.pack("<II", 264, 1), b"\0" * 240, struct.pack("<f3f", 0.0, 1.0, 1.0, 1.0),
             struct.pack("<I", L)]
    for v in range(L):
        parts += [tp[v].tobytes(), struct.pack("<I", L), tp.tobytes()]
    parts += [struct.pack("<II", width, height), struct.pack("<II", u_planes[0].shape[1], 0),
              struct.pack("<3f", 0, 0, 0), np.eye(3, dtype=np.float32).tobytes()]
    for U, S in zip(u_planes, sxv_planes):
        K = U.shape[1]
        parts += [struct.pack("<B", data_size), struct.pack("<III", K, U.shape[0], S.shape[0]),
                  np.ones(K, dt).tobytes(), np.ascontiguousarray(U, dt).tobytes(),
                  np.ascontiguousarray(S, dt).tobytes()]
    return b"".join(parts)


def btf_file_item(svf, ctx, layout, W, H, steps, dev, K=48):
    """A 400x400-texel DFMF file (FP16 planes, K components per channel): each texel
    a convex mix of K synthetic prototype texels (U = the prototypes' samples, SxV =
    Dirichlet weights).  Timed: the GPU decode alone, and svf_fit_btf (decode +
    fit, default initial guess) over the whole file."""
    import torch

    L = layout.light_count
    N, T = L * L, W * H
    proto = torch.empty((K, N, 3), dtype=torch.float32, device=dev)
    ctx.synth_btf(SEED + 5, MIX, layout.lights_parabolic, 0, K, proto)
    proto = proto.cpu().numpy()
    rng = np.random.default_rng(SEED)
    wts = rng.dirichlet(np.full(K, 0.3), size=T).astype(np.float32)
    theta_phi = np.zeros((L, 2), np.float32)
    # the ring layout's angles: theta rings 0/15/.../75 degrees, phi uniform per ring
    i = 0
    for ring, count in zip(range(6), (1, 6, 12, 18, 20, 24)):
        for k in range(count):
            theta_phi[i] = (np.radians(15.0 * ring), 2 * np.pi * k / count)
            i += 1
    data = dfmf_bytes(theta_phi, W, H, [proto[:, :, c].T for c in range(3)], [wts] * 3)
    t0 = time.perf_counter()
    btf = svf.Btf(ctx, data)
    load_s = time.perf_counter() - t0
    out = torch.empty((T, N, 3), dtype=torch.float32, device=dev)
    btf.decode(out=out)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        btf.decode(out=out)
    torch.cuda.synchronize()
    dec_s = (time.perf_counter() - t0) / steps
    # the fit alone on the decoded samples resident in HBM: the same texels as svf_fit_btf fits
    dmaps = {k: torch.zeros(sh, dtype=torch.float32, device=dev) for k, sh in
             {"rmse": (T,), "diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4)}.items()}
    ctx.fit_texels(layout, out, T, 1, want=tuple(dmaps), out=dmaps, check=False)
    rs_res = ctx.fit_texels(layout, out, T, 1, want=tuple(dmaps), out=dmaps, check=False)[1]
    del out, dmaps
    torch.cuda.empty_cache()
    want = ("diffuse", "specular", "sigma", "basis", "rmse")
    btf.fit(layout=layout, want=want, check=False)
    t0 = time.perf_counter()
    maps, rs = btf.fit(layout=layout, want=want, check=False)
    fit_s = time.perf_counter() - t0
    btf.close()
    flops = 2.0 * 3 * K * N * T
    return {"workload": f"DFMF {W}x{H} texels, ring-81, FP16 planes, {K} components per channel "
                        f"({len(data) / 1e6:.1f} MB file)",
            "load_s": load_s,
            "decode": {"value": T / dec_s, "unit": "texels/s", "ms": dec_s * 1e3,
                       "output_gb_per_s": T * N * 3 * 4 / dec_s / 1e9, "tflops": flops / dec_s / 1e12,
                       "note": "FP32 samples; sums in the reference's order (bit-exact), so the FP32 pipe "
                               "runs 2 instructions per product"},
            "fit_btf": {"value": T / fit_s, "unit": "texels/s", "seconds": fit_s, "ms_device_fit": rs.ms_total,
                        "failed_texels": int(rs.failed_texels), "mean_rmse": float(maps["rmse"].mean()),
                        "mean_iterations": rs.iterations / T,
                        "note": "host wall time of svf_fit_btf (decode into FP32 chunks + the fit pipeline); "
                                "maps copied to host"},
            "fit_of_decoded_samples_in_hbm": {"value": T / (rs_res.ms_total / 1e3), "unit": "texels/s",
                                              "ms": rs_res.ms_total, "mean_iterations": rs_res.iterations / T,
                                              "note": "svf_fit_texels on the decoded samples: these texels are "
                                                      "mixtures of 48 prototypes, which the one-lobe model fits in "
                                                      "more LM iterations than the synthetic one-lobe texels"}}


def reference_ms_eval_rate(lp, bounces, threads=None, tasks=None):
    """The reference's multi-scattering evaluator (oracle/_ref, BRDFEvaluator with
    BounceCount) on all host threads: pair evaluations per second over `tasks`
    parameter vectors x all pairs of the layout."""
    import concurrent.futures as cf

    import oracle

    if not oracle.ref_available():
        raise RuntimeError("oracle/_ref/libtempest_ref.so is not built")
    threads = threads or os.cpu_count() or 1
    tasks = tasks or threads
    rng = np.random.default_rng(5)
    params = [np.array([0.05 + 0.4 * rng.random(), 0.05 + 0.4 * rng.random(), 0.5 + rng.random(), 0.2 * rng.random(),
                        *(0.6 * (rng.random(3) - 0.5))]) for _ in range(tasks)]
    oracle.ref_brdf_all_ms(params[0], lp[:4], bounces)   # load and bind first
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(threads) as ex:   # ctypes calls release the GIL
        list(ex.map(lambda p: oracle.ref_brdf_all_ms(p, lp, bounces), params))
    secs = time.perf_counter() - t0
    return tasks * lp.shape[0] ** 2 / secs, secs, threads


def multi_scattering_item(svf, ctx, steps, dev, bounces=2, render_texels=256, fit_texels=64):
    """The pseudo-volume multi-scattering BRDF (svbrdffit -m) on ring-81: rendering
    (svf_render_btf_ms) and the SVF_LSQ_MULTI_SCATTERING fit, against the
    reference's evaluator on the host cores."""
    import torch

    lp = svf.directions_ring81()
    N = lp.shape[0] ** 2
    rng = np.random.default_rng(11)
    T = render_texels
    sigma = (0.08 + 0.3 * rng.random((T, 2))).astype(np.float32)
    quat = rng.standard_normal((T, 4)).astype(np.float32)
    quat /= np.linalg.norm(quat, axis=1, keepdims=True)
    kd = (0.2 * rng.random(T)).astype(np.float32)
    ks = (0.5 + rng.random(T)).astype(np.float32)
    grey = lambda a: np.repeat(a[:, None], 3, 1)
    out = torch.zeros((T, N, 3), dtype=torch.float32, device=dev)
    ctx.render_btf_ms(lp, grey(kd), grey(ks), sigma, quat, bounces, out=out)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.render_btf_ms(lp, grey(kd), grey(ks), sigma, quat, bounces, out=out)
    torch.cuda.synchronize()
    r_s = (time.perf_counter() - t0) / steps
    # the fit: the first fit_texels rendered texels (grey albedos, Euler angles 0:
    # the truth is a zero of the model) from a perturbed start
    F = fit_texels
    quat0 = np.tile(np.array([0, 0, 0, 1], np.float32), (F, 1))
    lum_rgb = ctx.render_btf_ms(lp, grey(kd[:F]), grey(ks[:F]), sigma[:F], quat0, bounces)
    lum = np.ascontiguousarray(lum_rgb[:, :, 0])
    truth = np.stack([sigma[:F, 0], sigma[:F, 1], ks[:F], kd[:F], np.zeros(F), np.zeros(F), np.zeros(F)], 1)
    init = (truth * (1 + 0.2 * rng.standard_normal((F, 7)))).astype(np.float32)
    init[:, :4] = np.abs(init[:, :4]) + 1e-3
    init[:, 4:] = 0.05 * rng.standard_normal((F, 3))
    opts = svf.options(multi_scattering=bounces)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fo, fr, fst = ctx.lsq_fit_batch(lp, lum, init, opts)
    torch.cuda.synchronize()
    f_s = time.perf_counter() - t0
    r0 = ctx.lsq_fit_batch(lp, lum, init, svf.options(max_iterations=0, multi_scattering=bounces))[1]
    evals_per_texel = float((14 * fst["jacobians"] + fst["residuals"]).mean()) * N
    item = {"workload": f"ring-81 (6561 pairs), {bounces} bounces, 256 walks per evaluation (the fitter's evaluator)",
            "render": {"value": T * N / r_s, "unit": "pair evaluations/s", "texels": T, "ms": r_s * 1e3,
                       "texels_per_s": T / r_s, "note": "svf_render_btf_ms into device memory, RGB"},
            "fit": {"value": F / f_s, "unit": "texels/s", "texels": F, "seconds": f_s,
                    "mean_iterations": float(fst["iterations"].mean()),
                    "mean_jacobians": float(fst["jacobians"].mean()),
                    "mean_residual_evaluations": float(fst["residuals"].mean()),
                    "evaluations_per_texel": evals_per_texel, "evaluations_per_s": F * evals_per_texel / f_s,
                    "mean_rmse_start": float(r0.mean()), "mean_rmse": float(fr.mean()),
                    "note": "host wall time of svf_lsq_fit_batch (SVF_LSQ_MULTI_SCATTERING), slices on the host"}}
    try:
        rate, secs, thr = reference_ms_eval_rate(lp, bounces)
        item["reference_cpu"] = {"value": rate, "unit": "pair evaluations/s", "cores": thr, "seconds": secs,
                                 "kind": "reference",
                                 "fit_texels_per_s_estimate": rate / evals_per_texel,
                                 "sample": f"{thr} parameter vectors x 6561 pairs on {thr} threads; the fit estimate "
                                           f"divides by the GPU fit's evaluations per texel (the same LM)"}
    except Exception as e:  # the checker may be absent on a box without it built
        item["reference_cpu"] = {"value": None, "sample": f"unavailable: {e}"}
    return item


def summarize(line, parity):
    """The line items' headline figures in a few short keys."""
    def r3(x):
        return None if x is None else float(f"{x:.4g}")

    out = {"parity_vs_reference": parity}
    li = line.get("learned_init")
    if li and li.get("config3_1024x1024_fp16"):
        c3 = li["config3_1024x1024_fp16"]
        out["config3"] = {"speedup_vs_plain_gpu_lm": r3(c3["speedup"]),
                          "speedup_with_fallback": r3(c3.get("with_fallback", {}).get("speedup")),
                          "residual_ratio_mean": r3(c3["residual_ratio"]["mean"]),
                          "within_1pct_or_at_target": r3(c3["residual_ratio"].get("within_1pct_or_at_target")),
                          "residual_ratio_mean_with_fallback": r3(c3.get("with_fallback", {}).get("residual_ratio_mean")),
                          "normal_p90_deg": {"plain": r3(c3["plain"]["ground_truth_error"]["normal_deg"]["p90"]),
                                             "learned": r3(c3["learned"]["ground_truth_error"]["normal_deg"]["p90"]),
                                             "with_fallback": r3(c3.get("with_fallback", {}).get("normal_p90_deg"))}}
    b = line.get("batch_8_btfs")
    if b:
        out["config4"] = {"batch_texels_per_s": r3(b["value"]),
                          "per_btf_texels_per_s": {p["btf"]: r3(p.get("texels_per_s")) for p in b["per_btf"]},
                          "learned_residual_ratio_mean": {p["btf"]: r3(p["learned"]["residual_ratio_vs_plain"]["mean"])
                                                          for p in b["per_btf"]}}
    f = line.get("fib151_768x768")
    if f:
        out["config2"] = {"texels_per_s": r3(f["value"]), "fp64_check": f.get("fp64_check_summary")}
    m = line.get("multi_scattering")
    if m:
        ref = m.get("reference_cpu") or {}
        out["multi_scattering"] = {"render_evals_per_s": r3(m["render"]["value"]),
                                   "fit_texels_per_s": r3(m["fit"]["value"]),
                                   "reference_cpu_evals_per_s": r3(ref.get("value")),
                                   "reference_fit_texels_per_s_estimate": r3(ref.get("fit_texels_per_s_estimate"))}
    return out


def run_ours(args):
    import torch

    import tempestrenderer_b200 as svf

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    W, H = args.width, args.height
    T = W * H
    layout = ring81_mesh()
    L = layout.light_count
    N = L * L
    ctx = svf.Context(local)
    # this rank's shard of a larger synthetic BTF: texels [rank*T, (rank+1)*T)
    samples = torch.empty((T, N, 3), dtype=torch.float32, device=dev)
    truth = torch.empty((T, 16), dtype=torch.float32, device=dev)
    ctx.synth_btf(SEED, MIX, layout.lights_parabolic, rank * T, T, samples, truth=truth)
    torch.cuda.synchronize()
    maps = {k: torch.zeros(s, dtype=torch.float32, device=dev) for k, s in
            {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
             "params": (T, 7)}.items()}
    want = tuple(maps.keys())
    opts = svf.options(max_iterations=1024)

    def step():
        res, rs = ctx.fit_texels(layout, samples, W, H, opts=opts, want=want, out=maps, check=False)
        return rs

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    stats = []
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            stats.append(step())
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if dist:
        dist.barrier()
    ms = float(sum(s.ms_total for s in stats))
    ms_fit = float(sum(s.ms_fit for s in stats))
    ms_init = float(sum(s.ms_init for s in stats))
    ms_ndf = float(sum(s.ms_ndf for s in stats))
    ms_lum = float(sum(s.ms_luminance for s in stats))
    jac = sum(s.jacobians for s in stats)
    res = sum(s.residuals for s in stats)
    failed = sum(s.failed_texels for s in stats)
    t_max = ms
    if dist:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = world * T * args.steps / (t_max / 1e3)

    # the 11-parameter RGB fit on the same texels (an extra line item, not the headline)
    rgb_fit = None
    if args.rgb_steps > 0 and world == 1:
        ropts = svf.options(max_iterations=1024, rgb=True)
        rmaps = {k: torch.zeros(s, dtype=torch.float32, device=dev) for k, s in
                 {"diffuse": (T, 3), "specular": (T, 3), "sigma": (T, 2), "basis": (T, 4), "rmse": (T,),
                  "params": (T, 12)}.items()}
        ctx.fit_texels(layout, samples, W, H, opts=ropts, want=want, out=rmaps, check=False)
        rstats = [ctx.fit_texels(layout, samples, W, H, opts=ropts, want=want, out=rmaps, check=False)[1]
                  for _ in range(args.rgb_steps)]
        rms = float(sum(r.ms_total for r in rstats))
        rgb_fit = {"value": T * args.rgb_steps / (rms / 1e3), "unit": "texels/s",
                   "ms_per_step": rms / args.rgb_steps,
                   "phases_ms": {"luminance": sum(r.ms_luminance for r in rstats) / args.rgb_steps,
                                 "init": sum(r.ms_init for r in rstats) / args.rgb_steps,
                                 "lm": sum(r.ms_fit for r in rstats) / args.rgb_steps},
                   "mean_rgb_rmse": float(rmaps["rmse"].mean().item()),
                   "median_rgb_rmse": float(rmaps["rmse"].median().item()),
                   "model": "11-parameter RGB fit (kd rgb, ks rgb, sigma, orientation), FP16 RGB slabs, "
                            "started from the luminance fit (default initial guess) coloured by the average "
                            "chromaticity; init phase = NDF guess + luminance LM"}

    # e2e through the C ABI with pinned host buffers
    e2e = None
    if args.e2e_steps > 0:
        host_samples = torch.empty((T, N, 3), dtype=torch.float32, pin_memory=True)
        host_samples.copy_(samples)
        host_maps = {k: torch.zeros(v.shape, dtype=torch.float32, pin_memory=True) for k, v in maps.items()}
        ctx.fit_texels(layout, host_samples, W, H, opts=opts, want=want, out=host_maps, check=False)
        if dist:
            dist.barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record()
        for _ in range(args.e2e_steps):
            ctx.fit_texels(layout, host_samples, W, H, opts=opts, want=want, out=host_maps, check=False)
        ev1.record()
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        if dist:
            t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        h2d = host_samples.numel() * 4
        d2h = sum(v.numel() * 4 for v in host_maps.values())
        e2e = {"value": world * T * args.e2e_steps / e2e_s, "unit": "texels/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "steps": args.e2e_steps}
        del host_samples

    head_rmse = maps["rmse"].cpu().numpy()
    truth_np = truth.cpu().numpy()
    head_truth_err = param_error(maps["params"].cpu().numpy(), truth_np)
    learned = fib = batch = btf_file = refit = None
    if world == 1 and args.refit_steps > 0:
        # svbrdffit -j on the benchmark texels, from the headline fit's maps
        p_in, r_in = maps["params"].clone(), maps["rmse"].clone()
        ctx.refit_neighborhood(layout, samples, W, H, p_in, r_in, want=("rmse",))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.refit_steps):
            rm, rrs = ctx.refit_neighborhood(layout, samples, W, H, p_in, r_in, want=("rmse",))
        torch.cuda.synchronize()
        rs_s = (time.perf_counter() - t0) / args.refit_steps
        refit = {"value": T / rs_s, "unit": "texels/s", "seconds": rs_s,
                 "candidate_fits_per_s": 9 * T / rs_s, "mean_iterations_per_candidate": rrs.iterations / (9 * T),
                 "mean_rmse_before": float(head_rmse.mean()), "mean_rmse_after": float(rm["rmse"].mean()),
                 "improved_texels": float((rm["rmse"] < head_rmse).mean()),
                 "note": "host wall time of svf_refit_neighborhood: luminance, 9 candidate LM fits per texel in one "
                         "launch, selection, maps pass; inputs on the device, maps to host"}
    if world == 1 and args.mlp_steps > 0:
        learned = learned_init_item(svf, ctx, layout, samples, W, H, head_rmse, args.mlp_steps, dev, truth_np)
    if world == 1 and args.btf_steps > 0:
        btf_file = btf_file_item(svf, ctx, layout, W, H, args.btf_steps, dev)
    # the larger line items run in fresh contexts with the benchmark's buffers released
    ctx.close()
    del samples, maps
    torch.cuda.empty_cache()
    if world == 1 and args.fib_steps > 0:
        with svf.Context(local) as c2:
            fib = fib151_item(svf, c2, args.fib_steps, dev)
        torch.cuda.empty_cache()
    if world == 1 and args.batch_steps > 0:
        with svf.Context(local) as c2:
            batch = batch_item(svf, c2, args.batch_steps, dev)
        torch.cuda.empty_cache()
    ms_item = None
    if world == 1 and args.ms_steps > 0:
        with svf.Context(local) as c2:
            ms_item = multi_scattering_item(svf, c2, args.ms_steps, dev)
        torch.cuda.empty_cache()

    if rank == 0:
        props = torch.cuda.get_device_properties(dev)
        clk = clocks.summary()
        peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
        peaks = json.load(open(peaks_path)) if os.path.exists(peaks_path) else {}
        sm_mhz = clk["sm_mhz"] or peaks.get("clocks_under_load", {}).get("sm_mhz_median") or 1335.0
        fp32_peak = props.multi_processor_count * 128 * 2 * sm_mhz * 1e6 / 1e12   # TFLOP/s at the sampled clock
        lm_flops = N * (FLOPS_JACOBIAN_PASS * jac + FLOPS_RESIDUAL_PASS * res)
        achieved = lm_flops / (ms_fit / 1e3) / 1e12
        bf16_peak = peaks.get("bf16_tflops")
        ndf_alg = 2.0 * T * NDF_ROWS * N * args.steps               # one FP32 GEMM
        # the tensor cores multiply the operator's non-empty 256 x 64 tiles only, 3 BF16 products each
        ndf_tiles, ndf_tiles_total = stats[-1].ndf_tiles, stats[-1].ndf_tiles_total
        ndf_hw = 2.0 * T * 256 * 64 * ndf_tiles * 3 * args.steps
        ndf_ach = ndf_alg / (ms_ndf / 1e3) / 1e12 if ms_ndf > 0 else None
        cpu = parity = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                idx = parity_indices(T)
                rate, secs, thr, ref_rmse = reference_fit_rate(len(idx), indices=idx)
                cpu = {"value": rate, "unit": "texels/s", "cores": thr, "kind": "reference",
                       "sample": f"{len(idx)} texels spread evenly over the benchmark BTF (indices "
                                 f"linspace(0, {T - 1}, {len(idx)})), {thr} threads, {secs:.1f} s"}
                parity = dict(parity_block(head_rmse[idx], ref_rmse),
                              what="GPU RMSE / reference CPU RMSE per texel, the same texels (default init)")
            except Exception as e:  # the checker may be absent on a box without it built
                cpu = {"value": None, "unit": "texels/s", "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {
            "metric": METRIC, "value": value, "unit": "texels/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"svbrdffit texel loop, {W}x{H} texels per GPU, ring-81 layout (6561 pairs), "
                                   f"RGB FP32 in HBM, mix 20% near-diffuse/10% anisotropic, default init, LM 1024 max",
                       "texels_per_gpu": T, "l2": "inputs 12.6 GB per GPU, larger than L2",
                       "cuda_graph": ["launched directly", "recorded and launched", "replayed"][stats[-1].graph],
                       "parallelism": f"texel shards x{world}"},
            "roofline": {"bound": "fp32", "kernel": "lm_fit_kernel", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "traffic": LM_DRAM_BYTES_PER_TEXEL * T,
                         "traffic_source": "ncu dram bytes per texel (160x160-texel ring-81 capture) x texels",
                         "peak_source": f"derived: {props.multi_processor_count} SMs x 128 FP32 lanes x 2 x "
                                        f"{sm_mhz:.0f} MHz (sampled SM clock under load); MEASURED_PEAKS.json "
                                        f"has no FP32 figure"},
            "roofline_ndf": None if ndf_ach is None or not bf16_peak else {
                "bound": "tensor", "kernel": "ndf_tc_kernel", "achieved": ndf_ach, "peak": bf16_peak,
                "unit": "TFLOP/s", "frac": ndf_ach / bf16_peak, "peak_source": "measured (bf16_tflops, burst)",
                "hw_bf16_tflops": ndf_hw / (ms_ndf / 1e3) / 1e12,
                "hw_frac": ndf_hw / (ms_ndf / 1e3) / 1e12 / bf16_peak,
                "traffic": NDF_DRAM_BYTES_PER_TEXEL * T,
                "tiles": {"multiplied": ndf_tiles, "all": ndf_tiles_total},
                "note": "achieved counts the dense FP32 product (2 x texels x 3217 x 6561) that the tile-skipping "
                        "GEMM delivers; hw counts the 3 BF16 products over the non-empty 256 x 64 operator "
                        "tiles the tensor cores execute"},
            "phases_ms": {"luminance": ms_lum / args.steps, "init": ms_init / args.steps,
                          "ndf_gemm": ms_ndf / args.steps, "lm": ms_fit / args.steps},
            "lm_work": {"kernel_config": {"threads": stats[-1].lm_threads, "slots": stats[-1].lm_slots},
                        "jacobian_passes": jac / args.steps, "residual_passes": res / args.steps,
                        "failed_texels": failed, "mean_rmse": float(head_rmse.mean()),
                        "median_rmse": float(np.median(head_rmse)), "ground_truth_error": head_truth_err},
            "clocks": clk, "e2e": e2e, "rgb_fit": rgb_fit, "learned_init": learned, "fib151_768x768": fib,
            "batch_8_btfs": batch, "btf_file": btf_file, "refit_neighborhood": refit, "multi_scattering": ms_item,
            "gpu_launches": 4 * args.steps,
            "wall_s": wall, "cpu_baseline": cpu,
        }
        # short summaries last, so that a reader of the line's tail sees them
        line["summary"] = summarize(line, parity)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--width", type=int, default=WIDTH)
    ap.add_argument("--height", type=int, default=HEIGHT)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--rgb-steps", type=int, default=2, help="steps of the RGB fit line item (0: skip)")
    ap.add_argument("--mlp-steps", type=int, default=2, help="steps of the learned-initial-guess line item (0: skip)")
    ap.add_argument("--fib-steps", type=int, default=1, help="steps of the 768x768 Fibonacci-151 line item (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=1, help="calls of the 8-BTF batch line item (0: skip)")
    ap.add_argument("--btf-steps", type=int, default=3, help="decodes of the DFMF-file line item (0: skip)")
    ap.add_argument("--refit-steps", type=int, default=1, help="runs of the neighbourhood-refit line item (0: skip)")
    ap.add_argument("--ms-steps", type=int, default=1,
                    help="renders of the multi-scattering line item, which also times one fit (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
