"""Benchmark: Fisher-vector encoded descriptors/s at K=256, D=80.

Workload (the configuration the metric is quoted on): batched uneven Fisher
encoding -- 4,096 images with per-image descriptor counts ~ lognormal
(median 3,000, sigma 1.0) clipped to [200, 20,000] (about 19 M descriptors,
6 GB of float32 PCA-like descriptors N(0, diag((1+i)^-0.8)) resident in HBM),
a fixed seeded K=256 diagonal GMM, improved Fisher vectors (square root + L2)
of 40,960 floats per image.  One step = one batched encode of all images.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Each path (exact CUDA-core fp32, tensor-core FP32 = fp16x3, BF16, BF16 +
router) is timed with CUDA events on the launching stream.  The tensor-core
FP32 and BF16 paths run through a batched-encode plan (vlb200_fisher_plan_*):
its tile shapes are autotuned on the workload and one whole encode is
captured in a CUDA graph before the timed region, and each step replays the
graph; the other paths call vlb200_fisher_encode_batch_device.  The headline
`value` is the FP32-grade tensor-core path (the reference's float arithmetic
class); every path's rate and its Fisher vectors' relative error against the
FP64 GPU encodings of all images are reported beside it, with the BF16+router
to FP32 ratio the metric compares.  `e2e` times the same metric through the public API with
host buffers (pinned host -> device copy of the step's descriptors, encode,
device -> host copy of the encodings, all inside the timed region).
Under torchrun every rank encodes its own image set (replicas, weak scaling);
the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FV-encoded descriptors/s, K=256 D=80: plain FP32 vs BF16+router @ rel err≤1e-3"
K, D = 256, 80
NUM_IMAGES = 4096
FLAGS = 3  # VL_FISHER_FLAG_IMPROVED
PATHS = ["exact", "fp32", "bf16", "bf16_router"]


def workload_desc(total):
    return {"workload": "batched uneven improved-FV encode: 4096 images, counts ~ lognormal("
                        "median 3000, sigma 1.0) clipped [200, 20000], D=80 PCA-like float32, "
                        "K=256 fixed seeded GMM",
            "images": NUM_IMAGES, "descriptors": int(total), "K": K, "D": D,
            "l2": "inputs (6 GB) larger than L2; no flush"}


# --------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------- workload
def make_workload(rank, device):
    import torch
    from vlfeat_b200 import workloads as W
    counts = W.config2_counts(4096)[:NUM_IMAGES]
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    total = int(offs[-1])
    pr, mu, cv = W.fv_gmm(K, D, seed=11)
    g = torch.Generator(device=device)
    from vlfeat_b200.replicas import rank_data_seed
    g.manual_seed(rank_data_seed(rank))
    lam = torch.from_numpy(W.pca_lambdas(D).astype(np.float32)).to(device)
    x = torch.randn((total, D), generator=g, device=device, dtype=torch.float32)
    x.mul_(lam.sqrt()[None, :])
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
    return dict(x=x, offs=offs, priors=t(pr), means=t(mu), covs=t(cv), total=total,
                np_gmm=(pr, mu, cv))


def train_router(capi, wl, n_train=200_000, m=16, threshold=0.99):
    """Router for the BF16+router path: trained (untimed) on the full-E-step
    posteriors of the first n_train descriptors of the workload."""
    import torch
    from vlfeat_b200 import workloads as W
    from vlfeat_b200.router import Router, targets
    x = wl["x"][:n_train].contiguous()
    q = torch.zeros((n_train, K), device="cuda")
    capi.gmm_posteriors_device(q, wl["priors"], wl["means"], wl["covs"], x, "exact")
    tidx = torch.zeros((n_train, 8), dtype=torch.int32, device="cuda")
    tw = torch.zeros((n_train, 8), dtype=torch.float32, device="cuda")
    targets(q, tidx, tw)
    r = Router(D, K, hidden=(128,), seed=7)
    r.set_input_transform(np.zeros(D, np.float32),
                          (1.0 / np.sqrt(W.pca_lambdas(D))).astype(np.float32))
    r.train(x, tidx, tw, epochs=4, batch=1024, lr=2e-3)
    r.set_default(m=m, threshold=threshold)
    # Held-out rows: fallback fraction and missed posterior mass.
    xe = wl["x"][n_train:n_train + 100_000].contiguous()
    qf = torch.zeros((xe.shape[0], K), device="cuda")
    capi.gmm_posteriors_device(qf, wl["priors"], wl["means"], wl["covs"], xe, "exact")
    qc = torch.zeros_like(qf)
    fb = r.posteriors(qc, wl["priors"], wl["means"], wl["covs"], xe, m=m, threshold=threshold)
    qc0 = torch.zeros_like(qf)
    r.posteriors(qc0, wl["priors"], wl["means"], wl["covs"], xe, m=m, threshold=0.0)
    from vlfeat_b200.router import missed_mass
    report = {"router_m": m, "router_threshold": threshold,
              "router_fallback_fraction": fb / xe.shape[0],
              "router_missed_mass": missed_mass(qf, qc),
              "router_missed_mass_without_fallback": missed_mass(qf, qc0)}
    del q, tidx, tw, qf, qc, qc0
    return r, report


def router_sweep(capi, wl, router, enc, nt, ref, m=16, thresholds=(0.999, 0.99999, 1.0), steps=3):
    """The BF16+router path at fallback thresholds above the default 0.99:
    rate (CUDA events, batched call), Fisher-vector error over all images,
    and the fraction of rows that fall back (on 100,000 rows)."""
    import torch
    s = torch.cuda.current_stream()
    xe = wl["x"][:100_000].contiguous()
    qc = torch.zeros((xe.shape[0], K), device="cuda")
    out = {}
    for thr in thresholds:
        router.set_default(m=m, threshold=thr)
        fb = router.posteriors(qc, wl["priors"], wl["means"], wl["covs"], xe, m=m, threshold=thr)
        encode(capi, wl, enc, nt, "bf16_router", s)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            encode(capi, wl, enc, nt, "bf16_router", s)
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        err = rel_errs(enc, ref)
        err.pop("per_image")
        out[str(thr)] = {"value": wl["total"] / (ms * 1e-3), "ms_per_step": ms, "fallback_fraction": fb / xe.shape[0],
                         "rel_err_max": err["max"], "rel_err_p50": err["p50"],
                         "images_over_1e-3": err["images_over_1e-3"]}
    router.set_default(m=m, threshold=0.99)
    del qc
    return out


def encode(capi, wl, enc, nt, prec, stream):
    capi.fisher_encode_batch_device(enc, wl["means"], wl["covs"], wl["priors"], wl["x"], wl["offs"],
                                    FLAGS, prec, nt, stream)


PLAN_PATHS = ("fp32", "bf16")  # tensor-core paths: autotuned plan replayed as a CUDA graph


def make_encoder(capi, wl, x, enc, nt, prec, stream, config=None):
    """One encode of the workload on `stream`: returns (replay, eager, info).
    Tensor-core paths use a batched-encode plan bound to (x, enc, nt): tile
    shapes autotuned on the workload (or `config`), one encode captured as a
    CUDA graph, `replay` launches the graph and `eager` runs the plan's
    launches directly.  Other paths call the batched API."""
    if prec not in PLAN_PATHS:
        def run():
            encode(capi, dict(wl, x=x), enc, nt, prec, stream)
        return run, run, {"api": "vlb200_fisher_encode_batch_device", "cuda_graph": False}
    plan = capi.FisherPlan(D, K, wl["offs"], FLAGS, prec)
    plan.set_gmm(wl["means"], wl["covs"], wl["priors"])
    tuned = None
    if config is None:
        tuned = plan.autotune(enc, x, nt, stream=stream)
    else:
        plan.set_config(stream=stream, **config)
    plan.capture(enc, x, nt, stream=stream)
    info = {"api": "vlb200_fisher_plan (autotuned, CUDA graph)", "cuda_graph": True,
            "plan_config": plan.get_config(), "autotune_best_ms": tuned}

    def replay():
        plan.launch(stream=stream)

    def eager():
        plan.execute(enc, x, nt, stream=stream)
    replay.plan = plan  # keep the plan alive with its closures
    return replay, eager, info


def time_path(capi, run, steps, warmup, dist):
    import torch
    s = torch.cuda.current_stream()
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = capi.launch_count()
    e0.record(s)
    for _ in range(steps):
        run()
    e1.record(s)
    torch.cuda.synchronize()
    launches = capi.launch_count() - l0
    return e0.elapsed_time(e1) / steps, launches  # this rank's step time


def fp64_reference(capi, wl, n_images=None):
    """FP64 GPU encodings of every image of the workload (the library's exact
    double kernels through vl_fisher_encode(VL_TYPE_DOUBLE), which match
    VLFeat's double path to 1e-10), kept on the device as float64."""
    import torch
    pr, mu, cv = wl["np_gmm"]
    offs = wl["offs"]
    n_images = len(offs) - 1 if n_images is None else min(n_images, len(offs) - 1)
    mu64, cv64, pr64 = mu.astype(np.float64), cv.astype(np.float64), pr.astype(np.float64)
    out = torch.empty((n_images, 2 * K * D), dtype=torch.float64, device="cuda")
    step = 256
    for j0 in range(0, n_images, step):
        j1 = min(n_images, j0 + step)
        x = wl["x"][int(offs[j0]):int(offs[j1])].double().cpu().numpy()
        for j in range(j0, j1):
            e, _ = capi.fisher_encode(x[offs[j] - offs[j0]:offs[j + 1] - offs[j0]], mu64, cv64, pr64, FLAGS)
            out[j] = torch.from_numpy(e)
    return out


def rel_errs(enc, ref):
    """Per-image relative L2 error of the encodings against the FP64 ones
    (both on the device), summarised over all images."""
    import torch
    n = ref.shape[0]
    a = enc[:n].double()
    e = (a - ref).norm(dim=1) / ref.norm(dim=1).clamp_min(1e-30)
    e = e.cpu().numpy()
    return {"max": float(e.max()), "p50": float(np.median(e)), "p99": float(np.quantile(e, 0.99)),
            "images_over_1e-5": int((e > 1e-5).sum()), "images_over_1e-3": int((e > 1e-3).sum()),
            "images": int(n), "per_image": e}


# --------------------------------------------------------- CPU baseline
def cpu_baseline(wl, ref=None, budget_s=12.0, kind_pref="reference"):
    """VLFeat's own OpenMP CPU code (oracle/_ref) on a bounded sample of the
    same workload, all host threads; falls back to the C restatement.  With
    `ref` (the FP64 encodings), also the float path's own error against
    FP64 on the images it encoded: the accuracy floor of the reference's
    float arithmetic on this workload."""
    from oracle import oracle as O
    pr, mu, cv = wl["np_gmm"]
    offs = wl["offs"]
    cores = os.cpu_count() or 1
    try:
        impl = O.Reference(threads=cores)
        kind = "reference"
    except (FileNotFoundError, OSError):
        impl = O.Restatement()
        kind = "port"
    nimg_max = min(256, len(offs) - 1)
    x = wl["x"][: int(offs[nimg_max])].cpu().numpy()
    t0 = time.perf_counter()
    done_desc, j = 0, 0
    encs = []
    while j < nimg_max and (time.perf_counter() - t0) < budget_s:
        e, _ = impl.fisher(x[offs[j]:offs[j + 1]], mu, cv, pr, FLAGS)
        encs.append(e)
        done_desc += int(offs[j + 1] - offs[j])
        j += 1
    dt = time.perf_counter() - t0
    out = {"value": done_desc / dt, "unit": "descriptors/s", "cores": cores, "kind": kind,
           "sample": f"first {j} images ({done_desc} descriptors) of the workload, "
                     f"vl_fisher_encode(VL_TYPE_FLOAT, IMPROVED) per image, {dt:.1f} s"}
    if ref is not None and encs:
        # The float path's own error against FP64 on every image of the
        # workload (not timed): the same images the GPU paths are judged on.
        nall = len(offs) - 1
        e = np.zeros(nall)
        step = 256
        for j0 in range(0, nall, step):
            j1 = min(nall, j0 + step)
            xs = wl["x"][int(offs[j0]):int(offs[j1])].cpu().numpy()
            r = ref[j0:j1].cpu().numpy()
            for jj in range(j0, j1):
                enc = encs[jj] if jj < len(encs) else \
                    impl.fisher(xs[offs[jj] - offs[j0]:offs[jj + 1] - offs[j0]], mu, cv, pr, FLAGS)[0]
                e[jj] = np.linalg.norm(enc.astype(np.float64) - r[jj - j0]) / np.linalg.norm(r[jj - j0])
        out["float_rel_err_vs_fp64"] = {"max": float(e.max()), "p50": float(np.median(e)),
                                        "p99": float(np.quantile(e, 0.99)),
                                        "images_over_1e-5": int((e > 1e-5).sum()), "images": int(nall)}
    return out


# ------------------------------------------------------------- roofline
def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def roofline(capi, wl, run, prec):
    """Dominant kernel's achieved rate from live CUDA-event timing of every
    launch (library profiling) of `run` (one eager encode), against the
    measured peak."""
    import torch
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        src = "measured"
    except (OSError, ValueError):
        src = "fallback"
    hbm = peaks.get("hbm_gbs", 6650.0)
    bf16 = peaks.get("bf16_tflops", 1590.0)
    capi.profile_reset()
    capi.profile_enable(True)
    for _ in range(2):
        run()
    torch.cuda.synchronize()
    prof = capi.profile_read()
    capi.profile_enable(False)
    capi.profile_reset()
    if not prof:
        return None, {}
    name, (n, ms) = max(prof.items(), key=lambda kv: kv[1][1])
    total = wl["total"] * 2
    per_launch_s = ms / n / 1e3
    units = total / n  # descriptors per launch
    # Algorithmic work per descriptor of the dominant kernel.
    if "logp" in name or "estep" in name:
        flop = 4.0 * K * D  # [x, x^2] . [mu/s2, -1/(2 s2)]^T
    elif "stats" in name:
        flop = 4.0 * K * D  # q^T [x, x^2]
    else:
        flop = 8.0 * K * D
    achieved = units * flop / per_launch_s / 1e12
    peak = bf16 if prec in ("bf16", "bf16_router") else bf16 / 3.0
    shares = {k: round(v[1] / sum(x[1] for x in prof.values()), 4) for k, v in prof.items()}
    # DRAM traffic per launch: bytes per descriptor from the committed ncu
    # capture of the same kernel on a smaller case, scaled by descriptors per
    # launch (traffic grows in proportion to the rows processed).
    traffic = None
    try:
        tpd = json.load(open(os.path.join(ROOT, "profiles", "traffic_per_descriptor.json")))
        bpd = tpd.get(name, {}).get(prec)
        traffic = bpd * units if bpd else None
    except (OSError, ValueError):
        pass
    # The same kernel against the HBM roofline: algorithmic bytes (x read,
    # q written or read) per descriptor.
    alg_bytes = {"tc_estep_f16x3": 320 + (2 if prec != "fp32" else 4) * K,
                 "tc_stats_f16x2": 320 + 2 * K, "tc_stats_f16x3": 320 + 4 * K}.get(name)
    hbm_view = None
    if alg_bytes:
        gbs = units * alg_bytes / per_launch_s / 1e9
        hbm_view = {"achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                    "algorithmic_bytes_per_descriptor": alg_bytes}
    return ({"bound": "tensor", "kernel": name, "achieved": achieved, "peak": peak,
             "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
             "traffic_unit": "bytes per launch",
             "peak_source": f"{src} ({'bf16 burst' if peak == bf16 else 'bf16 burst / 3, FP32-equivalent'})",
             "algorithmic_flop_per_descriptor": flop, "launch_ms": per_launch_s * 1e3,
             "descriptors_per_launch": units, "hbm_view": hbm_view}, shares)


# -------------------------------------------------------------- e2e
def e2e(capi, wl, prec, config, steps=3):
    """Same metric through the public API from pinned host buffers: each step
    copies the descriptors host -> device, encodes them and copies the
    encodings device -> host, all inside the timed region.  Tensor-core paths
    call vlb200_fisher_plan_execute_host (the path's plan with the tuned
    configuration; the copies overlap the encode chunk by chunk); other paths
    copy, call the batched API and copy back."""
    import torch
    x_host = wl["x"].cpu().pin_memory()
    total = wl["total"]
    enc_host = torch.empty((NUM_IMAGES, 2 * K * D), dtype=torch.float32).pin_memory()
    nt_host = torch.empty(NUM_IMAGES, dtype=torch.int64).pin_memory()
    s = torch.cuda.current_stream()
    if prec in PLAN_PATHS:
        plan = capi.FisherPlan(D, K, wl["offs"], FLAGS, prec)
        plan.set_gmm(wl["means"], wl["covs"], wl["priors"])
        if config:
            plan.set_config(stream=s, **config)

        def step():
            plan.execute_host(enc_host, x_host, nt_host, stream=s)
        api = "vlb200_fisher_plan_execute_host"
    else:
        x_dev = torch.empty_like(wl["x"])
        enc = torch.empty((NUM_IMAGES, 2 * K * D), device="cuda")
        nt = torch.empty(NUM_IMAGES, dtype=torch.int64, device="cuda")

        def step():
            x_dev.copy_(x_host, non_blocking=True)
            encode(capi, dict(wl, x=x_dev), enc, nt, prec, s)
            enc_host.copy_(enc, non_blocking=True)
            nt_host.copy_(nt, non_blocking=True)
        api = "vlb200_fisher_encode_batch_device"
    step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        step()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"value": total / (ms / 1e3), "unit": "descriptors/s", "api": api,
            "h2d_bytes_per_step": int(total * D * 4),
            "d2h_bytes_per_step": int(NUM_IMAGES * (2 * K * D * 4 + 8)), "ms_per_step": ms}


def em_throughput(capi, iters=5, cpu=True, large=True):
    """EM iterations/s, reported beside the Fisher metric.

    Config 1 (N=1,000,000 SIFT-like descriptors, D=128, K=256, custom init,
    variance floor 1e-4 x max global variance) and config 0 (N=50,000, D=64,
    K=64) run EM on device-resident data through vlb200_gmm_em_device in the
    EXACT (CUDA cores) and the FP32 and BF16 modes (E-step GEMM and M-step
    statistics GEMM on the tensor cores).  An iteration is one
    E-step plus one M-step (T iterations run T+1 E-steps, as vl/gmm.c:1220-1308).
    Timing: wall clock around the blocking call, after one untimed run.  The
    reference arm is VLFeat's OpenMP EM (oracle/_ref) on all host cores on a
    100,000-row sample of config 1."""
    import torch
    from vlfeat_b200 import workloads as W
    out = {"timing": "wall clock around vlb200_gmm_em_device (blocking), after one untimed run"}
    cfgs = [("config1_sift_n1m_d128_k256", W.config1(N=1_000_000, K=256, iters=20), 20),
            ("config0_n50k_d64_k64", W.config0(), 10)]

    def trace_errors(g, ref):
        """Per-iteration relative L2 errors of the parameters (after t M-steps)
        and of the log-likelihood against the FP64 run."""
        tr, lt = g.param_trace(), g.ll_trace
        rt, rl = ref
        n = min(len(tr), len(rt))
        per = {"means": [], "covariances": [], "priors": [], "loglikelihood": []}
        for t in range(n):
            for i, k in enumerate(("means", "covariances", "priors")):
                per[k].append(float(np.linalg.norm(tr[t][i] - rt[t][i]) / np.linalg.norm(rt[t][i])))
            per["loglikelihood"].append(abs(lt[t] - rl[t]) / abs(rl[t]))
        return {"max": {k: max(v) for k, v in per.items()}, "per_iteration": per}

    for name, c, T in cfgs:
        x = torch.from_numpy(np.ascontiguousarray(c["data"])).cuda()
        N = int(x.shape[0])
        res = {"N": N, "D": c["D"], "K": c["K"], "max_iterations": T}

        def model(dt):
            g = capi.GMM(c["D"], c["K"], dt)
            g.set_initialization("custom")
            g.set_max_num_iterations(T)
            g.set_covariance_lower_bound(c["lower_bound"])
            g.set_means(c["means"])
            g.set_covariances(c["covs"])
            g.set_priors(c["priors"])
            return g
        # FP64 on the GPU (exact double kernels, the reference's double
        # formulation) from the same initialisation: the error reference.
        g64 = model(np.float64)
        g64.set_param_trace(True)
        t0 = time.perf_counter()
        g64.cluster(c["data"].astype(np.float64))
        res["fp64"] = {"ms_per_iteration": 1e3 * (time.perf_counter() - t0) / max(1, len(g64.ll_trace) - 1),
                       "timing": "wall clock incl. the host -> device copy of the double data",
                       "iterations": len(g64.ll_trace) - 1}
        ref64 = (g64.param_trace(), g64.ll_trace)
        del g64
        for prec in ("exact", "fp32", "bf16"):
            def run(trace=False):
                g = model(np.float32)
                g.set_param_trace(trace)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ll = g.em_device(x, prec)
                torch.cuda.synchronize()
                return g, ll, time.perf_counter() - t0
            gt, _, _ = run(trace=True)  # untimed: per-iteration parameters for the errors
            errs = trace_errors(gt, ref64)
            del gt
            g, ll, dt = run()
            its = max(1, len(g.ll_trace) - 1)
            res[prec] = {"iterations": its, "ms_per_iteration": 1e3 * dt / its,
                         "iterations_per_s": its / dt, "descriptor_iterations_per_s": N * its / dt,
                         "log_likelihood": ll, "restarts": g.num_restarts,
                         "rel_err_vs_fp64_max": errs["max"],
                         "rel_err_vs_fp64_per_iteration": errs["per_iteration"] if name.startswith("config1") else None,
                         "kernels": {"exact": "CUDA-core fp32 E-step and M-step",
                                     "fp32": "tcgen05 fp16x3 E-step, fp16x3 M-step statistics",
                                     "bf16": "tcgen05 fp16x3 E-step, fp16x2 M-step statistics"}[prec]}
        out[name] = res
        del x
    if cpu:
        from oracle import oracle as O
        c = cfgs[0][1]
        n = 100_000
        try:
            impl, kind = O.Reference(threads=os.cpu_count() or 1), "reference"
        except (FileNotFoundError, OSError):
            impl, kind = O.Restatement(), "port"
        t0 = time.perf_counter()
        impl.em(np.ascontiguousarray(c["data"][:n]), c["priors"], c["means"], c["covs"],
                c["lower_bound"], 2)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"kind": kind, "cores": os.cpu_count() or 1,
                               "sample": f"config 1, first {n} descriptors, 2 iterations of vl_gmm_cluster",
                               "descriptor_iterations_per_s": n * 2 / dt,
                               "ms_per_iteration": 1e3 * dt / 2}
    if large:
        out["config4_streamed_n20m_d128_k1024"] = em_config4(capi, cpu=cpu)
    return out


def em_config4(capi, N=20_000_000, K=1024, D=128, T=15, m=16, threshold=0.99, judge_every=5, cpu=True):
    """Config 4: streamed EM at N = 20,000,000 SIFT-like descriptors (10 GB
    resident), D = 128, K = 1,024, 15 iterations from a custom initialisation
    (1,024 seeded rows, unbiased global variance, uniform priors, variance
    floor 1e-4 x the largest global variance); the N x K posteriors are never
    resident (82 GB in fp32).  Runs: the plain FP32 path (fp16x3 tensor-core
    E-step and statistics); the BF16 path (fp16x3 E-step, one fp16 q part in
    the statistics); BF16 with router-pruned E-steps (MLP 128-256-256-1024,
    m = 16, full E-step below 0.99 predicted candidate mass, those rows
    gathered through the tensor-core E-step) and a full E-step
    every 5th iteration, which re-fits the router and judges its missed
    posterior mass.  All three reduce the M-step in f64.  The BF16 runs'
    final log-likelihood and parameters are compared with the FP32 run's."""
    import torch
    from vlfeat_b200 import workloads as W
    from vlfeat_b200.router import Router
    x = W.sift_like_device(N, D, seed=400)
    pr, mu, cv, lb = W.custom_init_device(x, K, seed=401)

    def model():
        g = capi.GMM(D, K, np.float32)
        g.set_initialization("custom")
        g.set_max_num_iterations(T)
        g.set_covariance_lower_bound(lb)
        g.set_means(mu)
        g.set_covariances(cv)
        g.set_priors(pr)
        return g

    def rel(a, b):
        return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))

    out = {"N": N, "D": D, "K": K, "max_iterations": T, "data": "SIFT-like, generated on the GPU (seed 400)",
           "timing": "wall clock around vlb200_gmm_em_stream_device (blocking)"}
    runs = {}
    for name, prec, use_router in (("fp32", "fp32", False), ("bf16", "bf16", False),
                                   ("bf16_router", "bf16", True)):
        r = None
        if use_router:
            r = Router(D, K, hidden=(256, 256), seed=5)
            xm = x[:1 << 20].mean(0).cpu().numpy()
            xs = x[:1 << 20].std(0).clamp_min(1e-3).cpu().numpy()
            r.set_input_transform(xm, (1.0 / xs).astype(np.float32))
        g = model()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ll = g.em_stream_device(x, prec, router=r, m=m, threshold=threshold, judge_every=judge_every)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        rep = g.stream_report()
        its = len(rep) - 1
        res = {"seconds": dt, "iterations": its, "ms_per_iteration": 1e3 * dt / max(1, its),
               "descriptor_iterations_per_s": N * its / dt, "log_likelihood": ll, "restarts": g.num_restarts,
               "e_step_ms": [round(row["ms"], 1) for row in rep]}
        if use_router:
            res["router"] = {"m": m, "threshold": threshold, "judge_every": judge_every,
                             "judged_missed_mass": {str(t): rep[t]["missed_mass"] for t in range(len(rep))
                                                    if rep[t]["judged"]},
                             "fallback_fraction": {str(t): rep[t]["fallback_rows"] / N for t in range(len(rep))
                                                   if rep[t]["routed"]}}
        runs[name] = (g, res)
        out[name] = res
        del r
    ga = runs["fp32"][0]
    for name in ("bf16", "bf16_router"):
        g = runs[name][0]
        out[name]["vs_fp32_path"] = {
            "log_likelihood_rel": abs(g.loglikelihood - ga.loglikelihood) / abs(ga.loglikelihood),
            "means_rel": rel(g.means, ga.means), "covariances_rel": rel(g.covariances, ga.covariances),
            "priors_rel": rel(g.priors, ga.priors)}
    out["bf16_router_vs_fp32_speed"] = out["fp32"]["seconds"] / out["bf16_router"]["seconds"]
    if cpu:
        from oracle import oracle as O
        n4 = 20_000
        try:
            impl, kind = O.Reference(threads=os.cpu_count() or 1), "reference"
        except (FileNotFoundError, OSError):
            impl, kind = O.Restatement(), "port"
        xs = x[:n4].cpu().numpy()
        t0 = time.perf_counter()
        impl.em(np.ascontiguousarray(xs), pr, mu, cv, lb, 1)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"kind": kind, "cores": os.cpu_count() or 1,
                               "sample": f"first {n4} descriptors, 1 iteration of vl_gmm_cluster",
                               "descriptor_iterations_per_s": n4 / dt}
    del runs, x
    torch.cuda.empty_cache()
    return out


def vlad_throughput(capi, wl, steps=3, warmup=1, cpu=True, budget_s=8.0):
    """VLAD (vl_vlad_encode, vl/vlad.c:163-242) of the Fisher workload's
    images with hard assignments to the GMM means (vector quantisation, the
    usual VLAD input), intra-normalised (VL_VLAD_FLAG_NORMALIZE_COMPONENTS,
    then the global L2).  The batched device call's output is bit-equal to
    the reference; timed with CUDA events on the launching stream, inputs
    (descriptors N x D and assignments N x K, float32) resident in HBM and
    larger than L2.  Algorithmic bytes: 4(D + K) per descriptor read plus
    4KD per image written."""
    import torch
    x, mu, offs = wl["x"], wl["means"], wl["offs"]
    N, nimg = int(x.shape[0]), len(offs) - 1
    lab = torch.empty(N, dtype=torch.int64, device="cuda")
    mu2 = (mu * mu).sum(1)
    for i in range(0, N, 1 << 20):
        xb = x[i:i + (1 << 20)]
        lab[i:i + (1 << 20)] = (mu2[None, :] - 2.0 * xb @ mu.T).argmin(1)
    a = torch.zeros((N, K), dtype=torch.float32, device="cuda")
    a.scatter_(1, lab[:, None], 1.0)
    del lab
    flags = capi.VLAD_NORMALIZE_COMPONENTS
    enc = torch.empty((nimg, K * D), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        capi.vlad_encode_batch_device(enc, mu, x, a, offs, flags)
    torch.cuda.synchronize()
    ms = []
    l0 = capi.launch_count()
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        capi.vlad_encode_batch_device(enc, mu, x, a, offs, flags)
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    launches = (capi.launch_count() - l0) // steps
    t = float(np.median(ms))
    capi.profile_reset()
    capi.profile_enable(True)
    capi.vlad_encode_batch_device(enc, mu, x, a, offs, flags)
    torch.cuda.synchronize()
    prof = capi.profile_read()
    capi.profile_enable(False)
    capi.profile_reset()
    tot = sum(v[1] for v in prof.values()) or 1.0
    shares = {k: {"launches": int(v[0]), "ms": round(v[1], 4), "share": round(v[1] / tot, 4)}
              for k, v in prof.items()}
    alg = 4.0 * (D + K) * N + 4.0 * K * D * nimg
    peak = measured_peaks().get("hbm_gbs")
    out = {"workload": f"{nimg} images, {N} descriptors, D={D}, K={K}, hard assignments (nearest mean), "
                       "flags NORMALIZE_COMPONENTS", "ms_per_step": t, "value": N / (t * 1e-3),
           "unit": "descriptors/s", "gpu_launches": launches, "kernels": shares,
           "hbm": {"algorithmic_bytes": alg, "achieved_gbs": alg / (t * 1e-3) / 1e9, "peak_gbs": peak,
                   "frac": (alg / (t * 1e-3) / 1e9 / peak) if peak else None}}
    if cpu:
        from oracle import oracle as O
        try:
            impl = O.Reference(threads=os.cpu_count() or 1)
        except (FileNotFoundError, OSError):
            impl = None
        if impl is not None:
            j, done, same = 0, 0, 0
            xs = x[: int(offs[min(nimg, 256)])].cpu().numpy()
            as_ = a[: int(offs[min(nimg, 256)])].cpu().numpy()
            mun = mu.cpu().numpy()
            got = enc[:min(nimg, 256)].cpu().numpy()
            t0 = time.perf_counter()
            while j < min(nimg, 256) and time.perf_counter() - t0 < budget_s:
                r = impl.vlad(xs[offs[j]:offs[j + 1]], mun, as_[offs[j]:offs[j + 1]], flags)
                same += int(np.array_equal(r.view(np.uint32), got[j].view(np.uint32)))
                done += int(offs[j + 1] - offs[j])
                j += 1
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {"kind": "reference", "cores": os.cpu_count() or 1, "value": done / dt,
                                   "unit": "descriptors/s",
                                   "sample": f"first {j} images ({done} descriptors), vl_vlad_encode per image"}
            out["bit_exact_images"] = f"{same}/{j}"
    del a, enc
    torch.cuda.empty_cache()
    return out


def prologue_throughput(capi, wl, steps=3, warmup=1, cpu=True, budget_s=6.0):
    """The recognition app's descriptor prologue (apps/recognition/
    encodeImage.m:91-103) on the Fisher workload's images: 128-d descriptors ->
    P (x - c) with P 80 x 128 -> L2 renormalisation -> 'xy' extension with the
    frame normalised by its image's size (82-d output, the FV encoder's input
    in the app).  Inputs resident in HBM, CUDA events on the launching stream.
    The projection runs on the tensor cores in scaled fp16x3 (three MMAs per
    product).  Roofline: 848 B per descriptor of HBM traffic (the bound);
    2 x 128 x 80 flop per descriptor, three times that issued to the tensor
    cores, against the measured bf16 peak."""
    import torch
    offs = wl["offs"]
    N, nimg, din, dout = int(offs[-1]), len(offs) - 1, 128, 80
    g = torch.Generator(device="cuda")
    g.manual_seed(71)
    x = torch.rand((N, din), generator=g, device="cuda") * 255.0
    P = torch.randn((dout, din), generator=g, device="cuda") / 11.3
    c = torch.rand(din, generator=g, device="cuda") * 128.0
    sizes = torch.tensor([[640.0, 480.0]], device="cuda").repeat(nimg, 1)
    frames = torch.rand((N, 2), generator=g, device="cuda") * 400.0
    out = torch.empty((N, dout + 2), device="cuda")
    stream = torch.cuda.current_stream()
    run = lambda: capi.pca_project_device(out, x, P, c, True, frames, offs, sizes)
    for _ in range(warmup):
        run()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = float(np.median(ms))
    peaks = measured_peaks()
    flop = 2.0 * din * dout * N
    bytes_ = (4.0 * din + 8 + 4.0 * (dout + 2)) * N
    tpk = peaks.get("bf16_tflops")
    res = {"workload": f"{nimg} images, {N} descriptors, 128 -> 80 + xy, renormalised", "ms_per_step": t,
           "value": N / (t * 1e-3), "unit": "descriptors/s", "bound": "hbm",
           "hbm": {"achieved_gbs": bytes_ / (t * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                   "frac": bytes_ / (t * 1e-3) / 1e9 / peaks["hbm_gbs"] if peaks.get("hbm_gbs") else None,
                   "algorithmic_bytes_per_descriptor": 4.0 * din + 8 + 4.0 * (dout + 2)},
           "tensor": {"algorithmic_tflops": flop / (t * 1e-3) / 1e12,
                      "issued_tflops": 3 * flop / (t * 1e-3) / 1e12, "peak_tflops": tpk,
                      "frac_issued": 3 * flop / (t * 1e-3) / 1e12 / tpk if tpk else None}}
    if cpu:
        from oracle import oracle as O
        n = min(N, 2_000_000)
        xs, fs = x[:n].cpu().numpy(), frames[:n].cpu().numpy()
        Pn, cn = P.cpu().numpy(), c.cpu().numpy()
        t0 = time.perf_counter()
        done = 0
        while done < n and time.perf_counter() - t0 < budget_s:
            b = min(n - done, 250_000)
            O.pca_project(xs[done:done + b], Pn, cn, True, fs[done:done + b], np.array([0, b]),
                          np.array([[640.0, 480.0]]))
            done += b
        dt = time.perf_counter() - t0
        res["cpu_baseline"] = {"kind": "port", "cores": os.cpu_count() or 1, "value": done / dt,
                               "unit": "descriptors/s",
                               "sample": f"{done} descriptors through the float64 NumPy restatement "
                                         "(multithreaded BLAS); the reference's step is MATLAB"}
    del x, out, frames
    torch.cuda.empty_cache()
    return res


def kmeans_init_throughput(capi, cpu=True, n=1_000_000, n_cpu=25_000):
    """The GMM's KMeans initialisation (vl_gmm_init_with_kmeans, vl/gmm.c:
    1315-1370) on N = 1M rows of an 80-d, 256-component mixture (the shape
    of the Fisher workload's GMM training set), K = 256: random-selection
    seeding, ANN refinement (one kd-tree, N/4 comparisons, 5 iterations),
    exact assignment, one-hot M-step.  The call has host-side control flow
    (stopping tests, the kd-tree build over the K centres, random draws), so it
    is timed on the host clock around the C call with the device drained on
    both sides; the data is staged from host memory inside the timed call.
    The reference's time comes from a bounded sample (n_cpu rows), on which
    the GPU's assignments are also checked bit for bit."""
    import ctypes as C
    import torch
    from vlfeat_b200 import workloads as W
    x = W.mixture_data(n, 80, 256, seed=81)
    K, seed = 256, 811

    def run(xs):
        m = capi.GMM(xs.shape[1], K, np.float32)
        capi.rand_seed(seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        capi.lib().vl_gmm_init_with_kmeans(m._h, xs.ctypes.data_as(C.c_void_p), xs.shape[0], None)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        assert capi.lib().vl_get_last_error() == 0
        return m, dt

    run(x[:50_000])  # warm-up: kernels loaded, scratch sized
    capi.profile_reset()
    capi.profile_enable(True)
    l0 = capi.launch_count()
    m, dt = run(x)
    launches = capi.launch_count() - l0
    prof = capi.profile_read()
    capi.profile_enable(False)
    capi.profile_reset()
    del m
    tot = sum(v[1] for v in prof.values()) or 1.0
    shares = {k: {"launches": int(v[0]), "ms": round(v[1], 3), "share": round(v[1] / tot, 4)}
              for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:8]}
    out = {"workload": f"N={n} rows, D=80, K={K}, float32, vl_gmm_init_with_kmeans", "ms": 1e3 * dt,
           "value": n / dt, "unit": "rows/s", "gpu_launches": int(launches), "kernels": shares}
    # Dominant kernel: the brute-force screen, N x K x D elements per launch at
    # three separately rounded fp32 operations each (the reference's order, no
    # fused multiply-add), against the nominal fp32 issue rate of the CUDA cores.
    scr = prof.get("km_screen")
    if scr and scr[0] > 0:
        props = torch.cuda.get_device_properties(0)
        peak = props.multi_processor_count * 128 * measured_peaks().get("sm_max_mhz", 1965.0) * 1e6 / 1e12
        ach = 3.0 * n * K * 80 / (scr[1] / scr[0] * 1e-3) / 1e12
        out["roofline"] = {"kernel": "k_km_nearest (screen)", "bound": "fp32 issue", "achieved": ach,
                           "peak": peak, "unit": "T fp32 ops/s", "frac": ach / peak,
                           "ops_per_element": 3}
    if cpu:
        from oracle import oracle as O
        try:
            ref = O.Reference(threads=os.cpu_count() or 1)
        except (FileNotFoundError, OSError):
            ref = None
        if ref is not None:
            xs = np.ascontiguousarray(x[:n_cpu])
            t0 = time.perf_counter()
            r = ref.kmeans_init(xs, K, seed)
            dtc = time.perf_counter() - t0
            mg, dtg = run(xs)
            same = bool(np.array_equal(np.argmax(mg.posteriors, axis=1), r["assign"]))
            out["cpu_baseline"] = {"kind": "reference", "cores": 1, "value": n_cpu / dtc, "unit": "rows/s",
                                   "sample": f"first {n_cpu} rows, same K and seed; the reference's k-means "
                                             "runs single-threaded (its OpenMP clause does not compile "
                                             "with this GCC)"}
            out["gpu_on_sample"] = {"ms": 1e3 * dtg, "value": n_cpu / dtg, "bit_exact_assignments": same}
    torch.cuda.empty_cache()
    return out


def router_config3(capi, n_train=2_000_000, n_eval=10_000_000, ms=(4, 8, 16), threshold=0.99,
                   epochs=6, fv_images=1000, fv_rows=3000):
    """The learned router at its own configuration: K = 1,024, D = 80, a
    seeded 1,024-component mixture (sigma ~ U[0.3, 1.5]); an MLP 80 -> 256 ->
    256 -> 1024 (ReLU) trained by the library's own forward / backward / Adam
    kernels on the top-8 posteriors of the full E-step of 2,000,000
    descriptors, then evaluated on 10,000,000 held-out descriptors at m in
    {4, 8, 16}: missed posterior mass without fallback, the fraction of rows
    whose predicted candidate mass is below 0.99 (those fall back to the full
    E-step) and the missed mass with that fallback, against the full E-step's
    posteriors; and the improved Fisher vectors of 1,000 held-out images of
    3,000 descriptors through the router path against the FP32 path."""
    import torch
    from vlfeat_b200 import workloads as W
    from vlfeat_b200.router import Router, missed_mass, targets
    K3, D3 = 1024, 80
    params = W.config3_params(K3, D3)
    pr, mu, cv = (torch.from_numpy(a).cuda() for a in params)
    out = {"workload": f"K={K3}, D={D3}, mixture sigma ~ U[0.3, 1.5]; MLP {D3}-256-256-{K3}; "
                       f"{n_train} training / {n_eval} held-out descriptors", "threshold": threshold}
    xtr = W.config3_data_device(n_train, params, seed=501)
    q = torch.empty((n_train, K3), device="cuda")
    capi.gmm_posteriors_device(q, pr, mu, cv, xtr, "fp32")
    tidx = torch.empty((n_train, 8), dtype=torch.int32, device="cuda")
    tw = torch.empty((n_train, 8), dtype=torch.float32, device="cuda")
    targets(q, tidx, tw)
    del q
    r = Router(D3, K3, hidden=(256, 256), seed=3)
    xm, xs = xtr.mean(0).cpu().numpy(), xtr.std(0).cpu().numpy()
    r.set_input_transform(xm, (1.0 / xs).astype(np.float32))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    loss = r.train(xtr, tidx, tw, epochs=epochs, batch=1024, lr=2e-3)
    torch.cuda.synchronize()
    out["training"] = {"epochs": epochs, "batch": 1024, "last_epoch_loss": loss,
                       "seconds": time.perf_counter() - t0}
    del xtr, tidx, tw
    xev = W.config3_data_device(n_eval, params, seed=502)
    chunk = 1 << 20
    per_m = {}
    for m in ms:
        mm0 = mm1 = 0.0
        fb = 0
        t_router = 0.0
        for i in range(0, n_eval, chunk):
            xb = xev[i:i + chunk]
            b = xb.shape[0]
            qf = torch.empty((b, K3), device="cuda")
            capi.gmm_posteriors_device(qf, pr, mu, cv, xb, "fp32")
            qc = torch.empty_like(qf)
            r.posteriors(qc, pr, mu, cv, xb, m=m, threshold=0.0)
            mm0 += missed_mass(qf, qc) * b
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            fb += r.posteriors(qc, pr, mu, cv, xb, m=m, threshold=threshold)
            torch.cuda.synchronize()
            t_router += time.perf_counter() - t1
            mm1 += missed_mass(qf, qc) * b
            del qf, qc
        per_m[str(m)] = {"missed_mass_without_fallback": mm0 / n_eval,
                         "fallback_fraction": fb / n_eval, "missed_mass_with_fallback": mm1 / n_eval,
                         "router_posteriors_rows_per_s": n_eval / t_router}
    out["eval"] = per_m
    # Fisher vectors of held-out images through the router path (m = 8).
    n_img = min(fv_images, n_eval // fv_rows)
    offs = np.arange(n_img + 1, dtype=np.int64) * fv_rows
    xi = xev[: n_img * fv_rows].contiguous()
    ref = torch.empty((n_img, 2 * K3 * D3), device="cuda")
    capi.fisher_encode_batch_device(ref, mu, cv, pr, xi, offs, FLAGS, "fp32")
    enc = torch.empty_like(ref)
    fv = {}
    for m in ms:
        r.set_default(m=m, threshold=threshold)
        capi.fisher_encode_batch_device(enc, mu, cv, pr, xi, offs, FLAGS, "bf16_router")
        e = ((enc.double() - ref.double()).norm(dim=1) / ref.double().norm(dim=1)).cpu().numpy()
        fv[str(m)] = {"max": float(e.max()), "p50": float(np.median(e)), "images": int(n_img)}
    out["fv_rel_err_vs_fp32_path"] = fv
    capi.lib().vlb200_router_set_default(None, 8, 0.99)
    del r, xev, xi, ref, enc
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank, world):
    """The reference arm: VLFeat's own CPU code on the host cores."""
    if rank != 0:
        return
    from oracle import oracle as O
    from vlfeat_b200 import workloads as W
    counts = W.config2_counts(NUM_IMAGES)
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    pr, mu, cv = W.fv_gmm(K, D, seed=11)
    cores = os.cpu_count() or 1
    try:
        impl = O.Reference(threads=cores)
        kind = "reference"
    except (FileNotFoundError, OSError):
        impl = O.Restatement()
        kind = "port"
    nimg = 16  # images per step: a bounded sample of the workload
    x = W.pca_like(int(offs[nimg]), D, seed=301)
    times = []
    for it in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for j in range(nimg):
            impl.fisher(x[offs[j]:offs[j + 1]], mu, cv, pr, FLAGS)
        if it >= args.warmup:
            times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    v = int(offs[nimg]) / (ms / 1e3)
    sample = f"first {nimg} images ({int(offs[nimg])} descriptors) per step, vl_fisher_encode per image"
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "descriptors/s",
                      "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                      "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": workload_desc(int(offs[-1])),
                      "cpu_baseline": {"value": v, "unit": "descriptors/s", "cores": cores,
                                       "kind": kind, "sample": sample},
                      "e2e": {"value": v, "unit": "descriptors/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--paths", default=",".join(PATHS))
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-em", action="store_true", help="skip the EM iterations/s measurement")
    ap.add_argument("--no-vlad", action="store_true", help="skip the VLAD descriptors/s measurement")
    ap.add_argument("--no-prologue", action="store_true",
                    help="skip the descriptor prologue (PCA projection) measurement")
    ap.add_argument("--no-kmeans", action="store_true",
                    help="skip the GMM KMeans-initialisation measurement")
    ap.add_argument("--no-router-eval", action="store_true",
                    help="skip the learned router's evaluation at K=1024 (train 2M, evaluate 10M)")
    ap.add_argument("--router-train", type=int, default=2_000_000,
                    help="training descriptors of the router evaluation (smaller for profiling cases)")
    ap.add_argument("--router-eval", type=int, default=10_000_000,
                    help="held-out descriptors of the router evaluation (smaller for profiling cases)")
    ap.add_argument("--images", type=int, default=4096,
                    help="encode only the first IMAGES images of the workload (small profiling cases)")
    ap.add_argument("--plan", default=None,
                    help="fixed plan configuration instead of autotuning, e.g. "
                         "item_rows=4096,row_budget=0 (keys of FisherPlan.get_config)")
    args = ap.parse_args()
    global NUM_IMAGES
    NUM_IMAGES = args.images

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    from vlfeat_b200 import capi, replicas
    capi.lib()
    dev = torch.device("cuda")
    # All timing uses one explicit stream shared by torch and the library.
    torch.cuda.set_stream(torch.cuda.Stream())
    wl = make_workload(rank, dev)
    enc = torch.empty((NUM_IMAGES, 2 * K * D), device=dev)
    nt = torch.empty(NUM_IMAGES, dtype=torch.int64, device=dev)

    ref = fp64_reference(capi, wl) if rank == 0 else None
    router, router_report = None, {}
    if "bf16_router" in args.paths:
        router, router_report = train_router(capi, wl)
    results = {}
    launches_of = {}
    eager_of = {}
    s = torch.cuda.current_stream()
    encoders = {}
    fixed = None
    if args.plan:
        fixed = {k: int(v) for k, v in (kv.split("=") for kv in args.plan.split(","))}
    for p in args.paths.split(","):  # plans: autotuned and captured before the timed regions
        encoders[p] = make_encoder(capi, wl, wl["x"], enc, nt, p, s, config=fixed)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for p in args.paths.split(","):
            run, eager, info = encoders[p]
            ms_rank, launches = time_path(capi, run, args.steps, args.warmup, dist)
            value, ms = replicas.whole_job_rate(wl["total"], ms_rank, dist)  # max over ranks
            err = rel_errs(enc, ref) if rank == 0 else None
            results[p] = {"value": value, "ms_per_step": ms, "rel_err_vs_fp64": err, **info}
            if err is not None:
                err.pop("per_image")
            launches_of[p] = launches
            eager_of[p] = eager
    # The headline is the FP32-grade tensor-core path (fp16x3 split on both
    # contractions, fp32 accumulation): the reference's float arithmetic class.
    head = "fp32" if "fp32" in results else next(iter(results))
    if rank == 0:
        roof, shares = roofline(capi, wl, eager_of[head], head)
        peaks = measured_peaks()
        fp32_peak = peaks.get("bf16_tflops", 1590.0) / 3.0
        step_tflops = 8.0 * K * D * wl["total"] / (results[head]["ms_per_step"] * 1e-3) / 1e12
        out = {"metric": METRIC, "value": results[head]["value"], "unit": "descriptors/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": results[head]["ms_per_step"], "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None,
               "dtype": {"exact": "f32", "fp32": "f16x3", "bf16": "f16", "bf16_router": "f16"}[head],
               "precision_note": "f16x3: each operand split into two power-of-two-scaled fp16 parts "
                                 "(22 bits), three MMAs per product, fp32 accumulation (FP32-grade)",
               "data": "synthetic", "headline_path": head, "config": workload_desc(wl["total"]),
               "paths": results, "roofline": roof, "kernel_time_share": shares,
               "path_roofline": {"bound": "tensor", "algorithmic_flop_per_descriptor": 8.0 * K * D,
                                 "achieved": step_tflops, "peak": fp32_peak, "unit": "TFLOP/s",
                                 "frac": step_tflops / fp32_peak,
                                 "peak_source": "bf16 burst / 3 (FP32-equivalent tensor roofline)"},
               "gpu_launches": launches_of[head], "clocks": clk.summary()}
        # Flat keys: every path's rate and error, and the metric's comparison.
        for p, r in results.items():
            out[f"{p}_value"] = r["value"]
            out[f"{p}_rel_err_max"] = r["rel_err_vs_fp64"]["max"]
            out[f"{p}_rel_err_p50"] = r["rel_err_vs_fp64"]["p50"]
        if "bf16_router" in results and "fp32" in results:
            out["bf16_router_vs_fp32"] = results["bf16_router"]["value"] / results["fp32"]["value"]
            out["bf16_router_within_1e-3"] = results["bf16_router"]["rel_err_vs_fp64"]["max"] <= 1e-3
        if "bf16" in results and "fp32" in results:
            out["bf16_vs_fp32"] = results["bf16"]["value"] / results["fp32"]["value"]
        if router is not None:
            out.update(router_report)
            out["router_threshold_sweep"] = router_sweep(capi, wl, router, enc, nt, ref)
        if not args.no_e2e:
            out["e2e"] = e2e(capi, wl, head, results[head].get("plan_config"))
        if not args.no_cpu and world == 1:
            out["cpu_baseline"] = cpu_baseline(wl, ref)
            fe = out["cpu_baseline"].get("float_rel_err_vs_fp64")
            if fe:
                out["vlfeat_float_rel_err_max"] = fe["max"]
                out["vlfeat_float_rel_err_p50"] = fe["p50"]
        if not args.no_em and world == 1:
            del encoders, eager_of
            torch.cuda.empty_cache()
            out["em"] = em_throughput(capi, cpu=not args.no_cpu)
        if not args.no_vlad and world == 1:
            out["vlad"] = vlad_throughput(capi, wl, cpu=not args.no_cpu)
        if not args.no_prologue and world == 1:
            out["prologue"] = prologue_throughput(capi, wl, cpu=not args.no_cpu)
        if not args.no_kmeans and world == 1:
            out["kmeans_init"] = kmeans_init_throughput(capi, cpu=not args.no_cpu)
        if not args.no_router_eval and world == 1:
            if router is not None:
                capi.lib().vlb200_router_set_default(None, 8, 0.99)
                del router
            out["router_config3"] = router_config3(capi, n_train=args.router_train, n_eval=args.router_eval)
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
