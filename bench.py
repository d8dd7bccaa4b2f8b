"""Benchmark of the CY3 quintic metric-solver hot path on B200.

Workload (one GPU): Dwork quintic sum z^5 - 5 psi prod z, psi = 0.5, degree k = 6 with the ideal-reduced
section basis (N = 205), 500,000 line-intersection points; a step is one Donaldson balancing iteration
(T-operator, FP64 inverse, h update).  `value` is balancing iterations per second with the points and
section tables resident in HBM; `e2e` is the same metric through the C ABI from host buffers (points,
weights and log|Omega|^2 uploaded from pinned memory, h_block read back); sigma evaluations per second
and the FP64 path's iterations per second are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp16x3|bf16x3|fp64] [--impl reference]

Under torchrun each rank runs an independent replica on its own GPU (the path has no exchange step);
times are device times (CUDA events) and the max over ranks is reported.
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

METRIC = "balancing iters/s & sigma evals/s at k=6, 500k pts vs FP64; p50/p99 solve lat"
UNIT = "iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=os.environ.get("CY3Q_BENCH_PRECISION", "fp16x3"))
    ap.add_argument("--k", type=int, default=6)
    ap.add_argument("--points", type=int, default=500_000)
    ap.add_argument("--psi", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--sigma-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=256, help="0 skips the serving stream")
    ap.add_argument("--serving-rate", type=float, default=50.0)
    ap.add_argument("--serving-active", type=int, default=8)
    ap.add_argument("--galerkin-points", type=int, default=1_000_000, help="0 skips the Laplacian / Yukawa run")
    ap.add_argument("--adam-points", type=int, default=2_000_000, help="0 skips the sigma-Adam run")
    ap.add_argument("--adam-steps", type=int, default=200)
    ap.add_argument("--ty-points", type=int, default=40_000, help="0 skips the Tian-Yau and Schoen solves")
    ap.add_argument("--adam-minibatch", type=int, default=200_000)
    ap.add_argument("--traffic-csv", default=None,
                    help="ncu --page raw --csv export with dram__bytes_read.sum / dram__bytes_write.sum of the two "
                         "tensor-core kernels; their per-point DRAM bytes replace the built-in figures")
    ap.add_argument("--traffic-points", type=int, default=100096, help="padded points of the --traffic-csv capture")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clock and clock-event reasons of this process's GPU, sampled every 1 ms through NVML (the GPU found by
    its UUID, so the index does not depend on CUDA_VISIBLE_DEVICES); nvidia-smi at 200 ms when NVML is not
    available.  Reasons are kept when they were active in any sample."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.nvml = None
        self.lines: list[str] = []
        self.samples: list[tuple[float, int]] = []
        self.smax = None
        self._stop = threading.Event()

    def start(self):
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            uuid = "GPU-" + str(torch.cuda.get_device_properties(self.idx).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nvml = (pynvml, h)
            self._t = threading.Thread(target=self._poll, daemon=True)
            self._t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None

    def _poll(self):
        pynvml, h = self.nvml
        while not self._stop.is_set():
            try:
                self.samples.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                                     int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))))
            except Exception:
                pass
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.nvml is not None:
            self._stop.set()
            self._t.join(timeout=5)
            pynvml = self.nvml[0]
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            sm = [c for c, _ in self.samples]
            reasons = sorted({nm for _, r in self.samples for nm, bit in bits.items() if r & bit})
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(sm), "source": "nvml, 1 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(self.NAMES, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ------------------------------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def traffic_from_csv(path, pts):
    """Per-point DRAM bytes of umma_bergman_kernel / umma_gram_kernel from an ncu raw CSV export (ncu -i ...
    --page raw --csv) of a capture over `pts` padded points."""
    import csv

    rows = list(csv.reader(open(path)))
    hdr = rows[0]
    try:
        ik, ir, iw = hdr.index("Kernel Name"), hdr.index("dram__bytes_read.sum"), hdr.index("dram__bytes_write.sum")
    except ValueError:
        return None, None
    unit = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}
    u = rows[1]
    out = {}
    for r in rows[2:]:
        for stage, name in (("bergman", "umma_bergman_kernel"), ("toperator", "umma_gram_kernel")):
            if name in r[ik] and stage not in out:
                out[stage] = (float(r[ir]) * unit.get(u[ir], 1.0) + float(r[iw]) * unit.get(u[iw], 1.0)) / pts
    if len(out) != 2:
        return None, None
    return out, f"DRAM bytes per launch from {os.path.basename(path)} ({pts} points), scaled in points"


def algorithmic(P, N):
    return {
        "F_bal": 16.0 * P * N * N,          # 8PN^2 (K = s^H h s) + 8PN^2 (T = S^H W S)
        "F_T": 8.0 * P * N * N,
        "F_K": 8.0 * P * N * N,
        "F_sigma": 48.0 * P * N * N + 248.0 * P * N,
    }


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def cpu_baseline(pts, w, lo, k, psi, reduced=True):
    """One balancing iteration of the FP64 oracle port on the host cores over every point of the workload
    (no scaling): per-point K threaded, the T-operator sum serial, as in the reference."""
    import oracle

    oracle.set_threads(os.cpu_count() or 1)
    o = oracle.OracleSolver(pts, w, lo, oracle.monomials(k, reduced), psi, k, with_derivs=False)
    t0 = time.perf_counter()
    o.donaldson_step()
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": oracle.threads(), "kind": "port",
            "sample": f"1 FP64 balancing iteration over all {len(pts)} points (k={k}, N={o.n_basis}), {dt:.2f} s; "
                      f"per-point K threaded, T-operator sum serial as in the reference"}


N_REDUCED = {2: 15, 3: 35, 4: 70, 5: 125, 6: 205, 7: 315, 8: 460}


def serving_stream(a, dev):
    """Config 5: Poisson arrivals (mean rate a.serving_rate / s), psi uniform in the unit disk, k uniform in
    {2..8}, P = min(10 N^2, 2,000,000), 10 balancing iterations each, split precision; continuous batching
    by the library's server.  The one-at-a-time FP64 reference times one FP64 solve per k and weights it by
    the request mix."""
    from papers_b200 import cy3q

    rng = np.random.default_rng(2026)
    reqs = []
    t = 0.0
    for i in range(a.serving_requests):
        t += rng.exponential(1.0 / a.serving_rate)
        k = int(rng.integers(2, 9))
        u, v = rng.random(), rng.random()
        psi = np.sqrt(u) * np.exp(2j * np.pi * v)
        reqs.append((t, dict(k=k, n_points=min(10 * N_REDUCED[k] ** 2, 2_000_000), seed=1000 + i, psi=psi,
                             iterations=10, precision=a.precision)))
    # one solve of each request shape first, so that the autotuner's per-shape choice is made on an idle
    # device (it is cached for the process) and not while the stream's solves run
    for k in sorted({r["k"] for _, r in reqs}):
        w = cy3q.QuinticSolver.new_with_psi_sz(k, min(10 * N_REDUCED[k] ** 2, 2_000_000), 1, 0.5, reduced_basis=True,
                                               precision=a.precision, with_derivs=False, device=dev)
        w.donaldson_step()
        w.close()
    srv = cy3q.Server(dev, 0, a.serving_active)
    t0 = time.perf_counter()
    tickets = []
    for at, r in reqs:
        d = at - (time.perf_counter() - t0)
        if d > 0:
            time.sleep(d)
        tickets.append(srv.submit(**r))
    failed = 0
    for tk in tickets:
        if srv.wait(tk, 600000).status != 0:
            failed += 1
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    # one-at-a-time FP64 reference on the same GPU
    per_k = {}
    for k in sorted({r["k"] for _, r in reqs}):
        n = min(10 * N_REDUCED[k] ** 2, 2_000_000)
        s = cy3q.QuinticSolver.new_with_psi_sz(k, n, 7, 0.5, reduced_basis=True, precision="fp64",
                                               with_derivs=False, device=dev)
        import torch
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(10):
            s.donaldson_step()
        per_k[k] = time.perf_counter() - t1
        s.close()
    fp64_total = sum(per_k[r["k"]] for _, r in reqs)
    iters = sum(r["iterations"] for _, r in reqs)
    return {"requests": len(reqs), "failed": failed, "arrival_rate_per_s": a.serving_rate,
            "max_active": a.serving_active, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "iters_per_s": st["iters_per_s"], "wall_s": wall, "hbm_peak_bytes": st["hbm_peak"],
            "fp64_one_at_a_time_iters_per_s": iters / fp64_total,
            "fp64_one_at_a_time_s_per_solve_by_k": {str(k): v for k, v in per_k.items()},
            "precision": a.precision}


def galerkin_run(a, dev, stream, h_block):
    """Config 4: Laplacian spectrum on the balanced k=6 metric of the timed run (its h), assembled over
    fresh line-intersection points in split precision and in FP64; 40 lowest eigenvalues; 3x3x3 Yukawa
    overlap from seeded CN(0,1) coefficients over the same points."""
    import torch

    import papers_b200

    g = papers_b200.QuinticSolver.new_with_psi_sz(a.k, a.galerkin_points, a.seed + 1000, complex(a.psi),
                                                  reduced_basis=True, precision=a.precision, with_derivs=True,
                                                  device=dev)
    g.set_stream(stream.cuda_stream)
    g.h_block = h_block
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        fn()  # warm: scratch pool, cuSOLVER workspace
        torch.cuda.synchronize()
        g.profile_read(reset=True)
        ev0.record(stream)
        out = fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return out, ev0.elapsed_time(ev1)

    g.profile(True)
    ev, ms_split = timed(lambda: g.laplacian(40, 2, reg=1e-12))
    st_split = {k: v[0] / max(v[1], 1) for k, v in g.profile_read(reset=True).items()}
    g.set_precision("fp64")
    ev64, ms_64 = timed(lambda: g.laplacian(40, 2, reg=1e-12))
    st_64 = {k: v[0] / max(v[1], 1) for k, v in g.profile_read(reset=True).items()}
    g.set_precision(a.precision)
    rng = np.random.default_rng(a.seed)
    coeffs = (rng.standard_normal((3, 225)) + 1j * rng.standard_normal((3, 225))) / np.sqrt(2.0)
    y, ms_y = timed(lambda: g.yukawa(coeffs))
    g.profile(False)
    P = g.n_points
    g.close()
    scale = np.maximum(np.abs(ev64), 1.0)
    scale[0] = 1.0
    nf = 225
    flops = 2.0 * P * (2 * nf) ** 2 * 4  # real Gram flops: mass (P rows) + stiffness (3P rows)
    return {"points": P, "n_functions": nf, "precision": a.precision, "ms": ms_split, "fp64_ms": ms_64,
            "speedup_vs_fp64": ms_64 / ms_split, "eig_max_rel_err_vs_fp64": float(np.max(np.abs(ev - ev64) / scale)),
            "eigs_lowest": [float(x) for x in ev[:6]], "eig_40": float(ev[-1]),
            "stage_ms": st_split, "fp64_stage_ms": st_64,
            "gram_tflops_algorithmic": flops / (st_split.get("galerkin_gram", float("nan")) / 1e3) / 1e12,
            "yukawa_ms": ms_y, "yukawa_abs_max": float(np.abs(y).max()), "yukawa_000": [y[0, 0, 0].real, y[0, 0, 0].imag],
            "coefficients": "CN(0,1), numpy default_rng(seed), 3 x 225"}


def adam_run(a, dev, stream):
    """Config 3: sigma-functional Adam on the k=8 reduced basis (N=460), psi=0.1+0.2i, 2,000,000 points,
    lr 1e-3, minibatch 200,000 drawn by a seeded permutation, from the h of five balancing steps.  The FP64
    arm runs 10 steps from the same h; sigma and the gradient norm at the final h are compared with FP64
    on a fixed 200,000-point subset."""
    import torch

    import papers_b200

    psi = 0.1 + 0.2j
    g = papers_b200.QuinticSolver.new_with_psi_sz(8, a.adam_points, a.seed + 2000, psi, reduced_basis=True,
                                                  precision=a.precision, with_derivs=False, device=dev)
    g.set_stream(stream.cuda_stream)
    for _ in range(5):
        g.donaldson_step()
    h0 = g.h_block
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        ev0.record(stream)
        out = fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return out, ev0.elapsed_time(ev1)

    g.profile(True)
    g.profile_read(reset=True)
    hist, ms = timed(lambda: g.sigma_refine_analytic(a.adam_steps, 1e-3, minibatch=a.adam_minibatch, seed=a.seed))
    stages = {k: v[0] / max(v[1], 1) for k, v in g.profile_read(reset=True).items()}
    g.profile(False)
    h_final = g.h_block
    n64 = min(10, a.adam_steps)
    g.set_precision("fp64")
    g.h_block = h0
    hist64, ms64 = timed(lambda: g.sigma_refine_analytic(n64, 1e-3, minibatch=a.adam_minibatch, seed=a.seed))
    pts, w, lo = g.get_points()
    P = g.n_points
    g.close()
    m = min(a.adam_minibatch, P)
    sub = papers_b200.QuinticSolver.from_points(8, pts[:m], w[:m], lo[:m], psi=psi, reduced_basis=True,
                                                precision="fp64", device=dev)
    sub.set_stream(stream.cuda_stream)
    sub.h_block = h_final
    l2_64, gr64, l1_64 = sub.sigma_squared_and_gradient()
    sub.set_precision(a.precision)
    l2_s, gr_s, l1_s = sub.sigma_squared_and_gradient()
    sub.close()
    h = np.asarray(hist)
    return {"points": P, "n_basis": 460, "steps": len(hist), "minibatch": a.adam_minibatch, "lr": 1e-3,
            "precision": a.precision, "ms": ms, "steps_per_s": len(hist) / (ms / 1e3),
            "fp64_steps_per_s": n64 / (ms64 / 1e3), "speedup_vs_fp64": (len(hist) / ms) / (n64 / ms64),
            "sigma_first": float(h[0]), "sigma_last": float(h[-1]),
            "history_rel_diff_vs_fp64_first_steps": float(np.max(np.abs(h[:n64] / np.asarray(hist64) - 1))),
            "at_final_h_on_subset": {"points": m, "sigma_l1_rel_err": abs(l1_s / l1_64 - 1),
                                     "sigma_l2sq_rel_err": abs(l2_s / l2_64 - 1),
                                     "grad_norm_rel_err": abs(np.linalg.norm(gr_s) / np.linalg.norm(gr64) - 1),
                                     "grad_rel_frobenius": float(np.linalg.norm(gr_s - gr64) / np.linalg.norm(gr64))},
            "stage_ms_per_call": stages}


def cicy_run(a, dev, cfg, warm_cfg, basis, sigma_fn, cpu: bool, record_s: float):
    """One complete-intersection solve (solve_ty_metric / solve_schoen_metric) at the reference's production
    setting through the public API: the device sampler, the balancing loop and the sigma passes, wall-clock
    around the call (it synchronises every iteration, as the reference's loop reads each residual).  The CPU
    side times the oracle's port on the same cloud for two full iterations (Donaldson + sigma, all host
    threads); `record_s` is the reference's own recorded time per seed for this setting."""
    import torch

    from papers_b200 import ty

    ty.solve_ty_metric(warm_cfg)  # warm: library kernels and cuSOLVER loaded
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = ty.solve_ty_metric(cfg)
    torch.cuda.synchronize()
    solve_s = time.perf_counter() - t0
    ws = ty.TyWorkspace(cfg)
    t0 = time.perf_counter()
    n = ws.sample()
    torch.cuda.synchronize()
    sample_ms = 1e3 * (time.perf_counter() - t0)
    t0 = time.perf_counter()
    for _ in range(5):
        ws.donaldson_step()
    step_ms = 1e3 * (time.perf_counter() - t0) / 5
    t0 = time.perf_counter()
    for _ in range(5):
        ws.sigma()
    sigma_ms = 1e3 * (time.perf_counter() - t0) / 5
    out = {"workload": f"N={r['n_basis']}, {n} pts, tol {cfg.donaldson_tol:g}", "solve_s": solve_s,
           "reference_record_s": record_s, "iterations": r["iterations_run"], "sigma_final": r["sigma_final"],
           "sigma_fs_identity": r["sigma_fs_identity"], "residual": r["final_donaldson_residual"],
           "sample_ms": sample_ms, "step_ms": step_ms, "sigma_ms": sigma_ms,
           "gpu_ms_per_iteration": step_ms + sigma_ms}
    if cpu:
        import oracle

        oracle.set_threads(os.cpu_count() or 1)
        c, o2, w = ws.points()
        vals = oracle.ty_sections(c, basis, derivs=False)
        h = np.eye(r["n_basis"], dtype=complex)
        t0 = time.perf_counter()
        for _ in range(2):
            h, _res = oracle.ty_donaldson_step(vals, w, h)
            sigma_fn(c, o2, w, h)
        cpu_iter_s = (time.perf_counter() - t0) / 2
        out.update({"cpu_s_per_iteration": cpu_iter_s, "cpu_threads": oracle.threads(),
                    "speedup_per_iteration": 1e3 * cpu_iter_s / (step_ms + sigma_ms)})
    ws.close()
    return out


def ty_run(a, dev, cpu: bool):
    """Tian-Yau k = 3 and k = 4 and Schoen (3, 3, 1) at 40,000 points, up to 100 iterations to 1e-6 (the reference's
    P5.10 production settings; its records for seed 42: 20.1 s (k = 3, CPU path), 114.5 s (k = 4, its GPU path,
    adaptive damping) and 3.8 s per seed).  The k = 4 solve has no CPU column (the oracle's sigma at N = 200 and
    40,000 points takes minutes)."""
    from papers_b200 import ty

    out = {}
    tyb = scb = None
    if cpu:  # the CPU columns time the oracle's port; the GPU columns do not use it
        import oracle

        tyb, scb = oracle.ty_basis(3), oracle.schoen_basis(3, 3, 1)
    cfg = ty.TyMetricConfig(k_degree=3, n_sample=a.ty_points, max_iter=100, donaldson_tol=1e-6, seed=a.seed, device=dev)
    warm = ty.TyMetricConfig(k_degree=3, n_sample=2000, max_iter=3, donaldson_tol=1e-6, seed=a.seed, device=dev)
    out["tian_yau"] = cicy_run(a, dev, cfg, warm, tyb,
                               lambda c, o2, w, h: __import__("oracle").ty_sigma(c, o2, w, 3, h), cpu, 20.11)
    cfg4 = ty.TyMetricConfig(k_degree=4, n_sample=a.ty_points, max_iter=100, donaldson_tol=1e-6, seed=a.seed,
                             device=dev)
    warm4 = ty.TyMetricConfig(k_degree=4, n_sample=2000, max_iter=1, donaldson_tol=1e-6, seed=a.seed, device=dev)
    out["tian_yau_k4"] = cicy_run(a, dev, cfg4, warm4, None, None, False, 114.49)
    # the reference's P5.10 ensemble at k = 3: 20 seeds of each candidate (its record: 405.7 s + 101.9 s)
    seeds = [42, 100, 12345, 7, 99, 1, 2, 3, 4, 5, 137, 271, 314, 666, 1000, 2024, 4242, 57005, 48879, 51966]
    import torch

    ens = {}
    for name, mk in (("ty", lambda sd: ty.TyMetricConfig(k_degree=3, n_sample=a.ty_points, max_iter=100,
                                                          donaldson_tol=1e-6, seed=sd, device=dev)),
                     ("schoen", lambda sd: ty.SchoenMetricConfig(n_sample=a.ty_points, max_iter=100,
                                                                 donaldson_tol=1e-6, seed=sd, device=dev))):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rs = ty.solve_many([mk(sd) for sd in seeds], workers=4)
        torch.cuda.synchronize()
        ens[name + "_s"] = time.perf_counter() - t0
        ens[name + "_sigma_final_median"] = float(np.median([r["sigma_final"] for r in rs]))
    ens.update({"seeds": len(seeds), "total_s": ens["ty_s"] + ens["schoen_s"], "reference_total_s": 507.67,
                "workers": 4})
    out["p5_10_ensemble"] = ens
    scfg = ty.SchoenMetricConfig(n_sample=a.ty_points, max_iter=100, donaldson_tol=1e-6, seed=a.seed, device=dev)
    swarm = ty.SchoenMetricConfig(n_sample=2000, max_iter=3, donaldson_tol=1e-6, seed=a.seed, device=dev)
    out["schoen"] = cicy_run(a, dev, scfg, swarm, scb,
                             lambda c, o2, w, h: __import__("oracle").schoen_sigma(c, o2, w, (3, 3, 1), h), cpu, 3.77)
    return out


def run_reference(a, ws, rank):
    """The reference's CPU path (its Rust crate cannot be built here: no toolchain and its first-party
    dependency pwos-math is absent), as the oracle's FP64 port of it, on the whole workload: the same
    500,000 points, W untimed and K timed Donaldson iterations, every host core."""
    if rank != 0:
        return
    import oracle

    oracle.build()
    # identical synthetic points to our arm (oracle sampler, same seed / psi)
    pts, _ = oracle.sample_sz(a.points, a.seed, a.psi, fermat_variant=False)
    w = oracle.weights(pts, a.psi)
    lo, _, _ = oracle.log_omega(pts, a.psi)
    oracle.set_threads(os.cpu_count() or 1)
    o = oracle.OracleSolver(pts, w, lo, oracle.monomials(a.k, True), a.psi, a.k, with_derivs=False)
    for _ in range(max(a.warmup, 0)):
        o.donaldson_step()
    o.h_block = np.eye(2 * o.n_basis)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        o.donaldson_step()
    dt = time.perf_counter() - t0
    v = a.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * dt / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Dwork psi={a.psi} k={a.k} reduced N={o.n_basis}, {len(pts)} line-intersection "
                                   f"points, one Donaldson iteration per step", "precision": "fp64",
                       "l2": "inputs larger than L2"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": oracle.threads(), "kind": "port",
                             "sample": f"{a.steps} timed iterations over all {len(pts)} points after {a.warmup} "
                                       f"untimed ones (oracle FP64 port of the reference Rust path)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def relaunch_under_torchrun(a):
    """`--gpus N` with N > 1 outside torchrun: start N ranks (one per GPU) the way the driver does."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    os.execv(sys.executable, cmd)


def main():
    a = parse()
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        relaunch_under_torchrun(a)
    ws, rank, local = dist_setup()
    if ws != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} does not match the {ws} ranks started by torchrun")
    if a.impl == "reference":
        run_reference(a, ws, rank)
        return
    import torch

    import papers_b200
    from papers_b200 import build as pbuild

    pbuild.build()
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    psi = complex(a.psi)
    # ---- sample set (untimed): GPU line-intersection sampler on this rank's GPU ----
    s = papers_b200.QuinticSolver.new_with_psi_sz(a.k, a.points, a.seed + rank, psi, reduced_basis=True,
                                                  precision=a.precision, with_derivs=True, device=dev)
    s.set_stream(stream.cuda_stream)
    P, N = s.n_points, s.n_basis
    # warm-up covers both paths of the timed region: the first step after an externally set h (one
    # refactorisation, whose library kernels load on first use) and the graph-replayed steps
    for i in range(a.warmup):
        if i == 0:
            s.h_block = np.eye(2 * N)
        s.donaldson_step()
    s.h_block = np.eye(2 * N)

    # ---- timed region: K balancing iterations, device-timed (the production path: each step's body is
    # replayed from a CUDA graph).  The clock record is sampled every 1 ms from just before the timed
    # region to its end (one 20-iteration solve at this workload takes about 25 ms) ----
    clk = ClockSampler(dev)
    s.launch_count(reset=True)
    barrier(ws)
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    residuals = [s.donaldson_step() for _ in range(a.steps)]
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1)
    launches = s.launch_count(reset=True)
    h_run = s.h_block
    ms_max = dist_max(ms, ws)
    value = ws * a.steps / (ms_max / 1e3)

    # ---- stage breakdown: the same K iterations again from h = I with per-stage CUDA events (eager
    # launches, so every stage boundary can be timed); gives the roofline kernel's launch duration ----
    s.h_block = np.eye(2 * N)
    s.profile(True)
    s.profile_read(reset=True)
    for _ in range(a.steps):
        s.donaldson_step()
    torch.cuda.synchronize()
    stages = s.profile_read(reset=True)
    s.profile(False)
    s.h_block = h_run

    # ---- sigma evaluations per second; the first call on a point set also builds the digit planes of its
    # section table (timed separately as setup) ----
    torch.cuda.synchronize()
    ev0.record(stream)
    s.sigma()
    ev1.record(stream)
    torch.cuda.synchronize()
    sigma_setup_ms = dist_max(ev0.elapsed_time(ev1), ws)
    s.profile(True)
    s.profile_read(reset=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    sig = None
    for _ in range(a.sigma_steps):
        sig = s.sigma()
    ev1.record(stream)
    torch.cuda.synchronize()
    sigma_ms = dist_max(ev0.elapsed_time(ev1), ws)
    sigma_per_s = ws * a.sigma_steps / (sigma_ms / 1e3)
    sigma_stages = {k: v[0] / max(v[1], 1) for k, v in s.profile_read(reset=True).items()}
    s.profile(False)

    # ---- FP64 plain path on the same points: the 10x denominator and the accuracy reference ----
    fp64_per_s, acc, sigma64_per_s = None, None, None
    if a.precision != "fp64":
        s.set_precision("fp64")
        s.h_block = np.eye(2 * N)
        s.donaldson_step()  # untimed: the FP64 path's first step takes its cuSOLVER handle and workspaces
        s.h_block = np.eye(2 * N)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(a.steps):
            s.donaldson_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        fp64_per_s = ws * a.steps / (dist_max(ev0.elapsed_time(ev1), ws) / 1e3)
        h64 = s.h_block
        sig64 = s.sigma()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(a.sigma_steps):
            s.sigma()
        ev1.record(stream)
        torch.cuda.synchronize()
        sigma64_per_s = ws * a.sigma_steps / (dist_max(ev0.elapsed_time(ev1), ws) / 1e3)
        # the split path's sigma at its own h against the FP64 pass at that same h (the sigma arithmetic alone)
        s.h_block = h_run
        sig64_same_h = s.sigma()
        acc = {"h_rel_frobenius": float(np.linalg.norm(h_run - h64) / np.linalg.norm(h64)),
               "sigma_fp64": sig64, "sigma_rel_err": abs(sig / sig64 - 1.0) if sig else None,
               "sigma_rel_err_same_h": abs(sig / sig64_same_h - 1.0) if sig else None,
               "iterations": a.steps}
        s.set_precision(a.precision)
        s.h_block = h_run
    else:
        fp64_per_s = value
        sigma64_per_s = sigma_per_s

    # ---- e2e through the C ABI from pinned host buffers ----
    pts, w, lo = s.get_points()
    hp = torch.from_numpy(pts).pin_memory()
    hw = torch.from_numpy(w).pin_memory()
    hl = torch.from_numpy(lo).pin_memory()
    e = papers_b200.QuinticSolver(a.k, 0, 0, psi, fermat_variant=False, reduced_basis=True, precision=a.precision,
                                  with_derivs=False, device=dev, sample=False)
    e.set_stream(stream.cuda_stream)
    h_out = np.empty((2 * N, 2 * N))

    def e2e_run():
        e.set_points(hp.numpy(), hw.numpy(), hl.numpy())
        for _ in range(a.steps):
            e.donaldson_step()
        e.get_h(out=h_out)

    e2e_run()  # warm: device buffers of the handle are allocated once and reused
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    ev0.record(stream)
    e2e_run()
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = dist_max(ev0.elapsed_time(ev1), ws)
    e2e_wall = dist_max(time.perf_counter() - t0, ws)
    e.close()
    h2d = (pts.nbytes + w.nbytes + lo.nbytes) / a.steps
    d2h = (h_out.nbytes + 8 * a.steps) / a.steps
    e2e_value = ws * a.steps / (e2e_ms / 1e3)

    # ---- roofline of the dominant stage ----
    # Per launch of each tensor-core kernel of the split step (ldk = 2N rounded up to 64, Pp = P rounded up
    # to 128): algorithmic flops 8 P N^2 (one complex contraction); algorithmic bytes: the Bergman kernel
    # reads the split section rows X (hi + lo, Pp ldk 4 B) and writes the split T-operand Xt (Pp ldk 4 B);
    # the T-operator reads Xt once (Pp ldk 4 B).  The binding roof is the one with the longer floor time
    # (bytes / measured HBM copy bandwidth vs. 3 split products x flops / measured bf16 burst).
    pk, src = peaks()
    alg = algorithmic(P, N)
    ldk = -(-2 * N // 64) * 64
    Pp = -(-P // 128) * 128
    stage_flops = {"toperator": alg["F_T"], "bergman": alg["F_K"]}
    stage_bytes = {"bergman": 2.0 * Pp * ldk * 4, "toperator": 1.0 * Pp * ldk * 4}
    # DRAM bytes per point of the two kernels (dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of
    # each kernel on the 100,096-point case of this workload, `--points 100000`), scaled in points: both stream
    # their operands once.  --traffic-csv reads the figures from an ncu --page raw --csv export instead.
    traffic_per_point, traffic_src = (traffic_from_csv(a.traffic_csv, a.traffic_points) if a.traffic_csv
                                      else (None, None))
    if traffic_per_point is None:
        traffic_per_point = {"bergman": (205.269504e6 + 121.626112e6) / 100096,
                             "toperator": (191.440640e6 + 13.993472e6) / 100096}
        traffic_src = "DRAM bytes per launch scaled from the 100,096-point ncu capture of these kernels"
    cand = {k: v for k, v in stages.items() if k in stage_flops}
    dname, (dms, dcalls) = max(cand.items(), key=lambda kv: kv[1][0]) if cand else ("toperator", (ms, a.steps))
    avg_ms = dms / max(dcalls, 1)
    if a.precision == "fp64":
        roof = {"bound": "fp64", "achieved": stage_flops[dname] / (avg_ms / 1e3) / 1e12, "peak": 37.0,
                "unit": "TFLOP/s", "peak_source": "nominal FP64 peak (MEASURED_PEAKS.json has no FP64 figure)",
                "traffic": None}
        roof["frac"] = roof["achieved"] / roof["peak"]
    else:
        hbm, tf = pk["hbm_gbs"], pk["bf16_tflops"]
        floor_hbm_ms = stage_bytes[dname] / (hbm * 1e9) * 1e3
        floor_tensor_ms = 3.0 * stage_flops[dname] / (tf * 1e12) * 1e3
        tensor_view = {"achieved": stage_flops[dname] / (avg_ms / 1e3) / 1e12, "peak": tf, "unit": "TFLOP/s",
                       "floor_ms": floor_tensor_ms,
                       "note": "algorithmic flops (8PN^2); the fp16x3 split runs 3 MMA products per flop, so "
                               "the ceiling of achieved / peak is 1/3"}
        tensor_view["frac"] = tensor_view["achieved"] / tf
        hbm_view = {"achieved": stage_bytes[dname] / (avg_ms / 1e3) / 1e9, "peak": hbm, "unit": "GB/s",
                    "floor_ms": floor_hbm_ms, "algorithmic_bytes_per_launch": stage_bytes[dname]}
        hbm_view["frac"] = hbm_view["achieved"] / hbm
        main = hbm_view if floor_hbm_ms >= floor_tensor_ms else tensor_view
        roof = {"bound": "hbm" if main is hbm_view else "tensor", "achieved": main["achieved"], "peak": main["peak"],
                "unit": main["unit"], "frac": main["frac"], "traffic": traffic_per_point[dname] * P,
                "peak_source": f"{src} (MEASURED_PEAKS.json: HBM copy GB/s, bf16 dense burst TF/s; each kernel runs "
                               f"< 1 ms)",
                "hbm_view": hbm_view, "tensor_view": tensor_view}
    roof.update({"kernel_stage": dname, "avg_launch_ms": avg_ms,
                 "kernel": {"bergman": "umma_bergman_kernel", "toperator": "umma_gram_kernel"}[dname],
                 "algorithmic_flops_per_launch": stage_flops[dname],
                 "traffic_note": traffic_src,
                 "stage_ms_per_step": {k: v[0] / max(v[1], 1) for k, v in stages.items()}})

    galerkin = None
    if a.galerkin_points > 0:
        barrier(ws)
        galerkin = galerkin_run(a, dev, stream, h_run)

    adam = None
    if a.adam_points > 0:
        barrier(ws)
        adam = adam_run(a, dev, stream)

    serving = None
    if a.serving_requests > 0:
        barrier(ws)
        try:
            serving = serving_stream(a, dev)
        except Exception as exc:  # the balancing line above is complete; report the failed section in it
            serving = {"error": f"{type(exc).__name__}: {exc}"[:500]}

    tian_yau = None
    if a.ty_points > 0:
        barrier(ws)
        try:
            tian_yau = ty_run(a, dev, cpu=rank == 0 and ws == 1 and not a.no_cpu_baseline)
        except Exception as exc:
            tian_yau = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(pts, w, lo, a.k, psi)

    if rank == 0:
        # the per-stage maps and the full section records go to stderr as one JSON object; the result line on
        # stdout keeps scalars, so that it stays short and the accuracy figures sit at its end
        detail = {"stage_ms_per_step": roof.pop("stage_ms_per_step", None), "hbm_view": roof.pop("hbm_view", None),
                  "tensor_view": roof.pop("tensor_view", None), "sigma_stage_ms": sigma_stages,
                  "laplacian": galerkin, "sigma_adam": adam, "serving": serving, "cicy": tian_yau}
        print("bench detail: " + json.dumps(detail), file=sys.stderr, flush=True)

        def pick(d, keys):
            return None if d is None else {k: d.get(k) for k in keys if k in d}

        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": a.steps, "warmup": a.warmup,
                "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if a.precision == "fp64" else a.precision, "data": "synthetic",
                "config": {"workload": f"Dwork psi={a.psi} k={a.k} N={N}, {P} pts, 1 balancing iteration/step",
                           "precision": a.precision, "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2 (section table %.2f GB)" % (P * 6 * (2 * N + 30) * 8 / 1e9)},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                        "wall_s": e2e_wall},
                "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
                "laplacian": pick(galerkin, ["ms", "fp64_ms", "eig_max_rel_err_vs_fp64", "yukawa_ms"]),
                "sigma_adam": pick(adam, ["steps_per_s", "fp64_steps_per_s"]) if adam else None,
                "sigma_adam_err": pick((adam or {}).get("at_final_h_on_subset"),
                                       ["sigma_l1_rel_err", "grad_rel_frobenius"]) if adam else None,
                "serving": pick(serving, ["error", "failed", "p50_ms", "p99_ms", "iters_per_s",
                                          "fp64_one_at_a_time_iters_per_s"]),
                "tian_yau": pick((tian_yau or {}).get("tian_yau", tian_yau),
                                 ["error", "solve_s", "iterations", "sigma_final", "gpu_ms_per_iteration",
                                  "cpu_s_per_iteration"]) if tian_yau else None,
                "schoen": pick((tian_yau or {}).get("schoen"), ["solve_s", "iterations", "sigma_final",
                                                               "gpu_ms_per_iteration", "cpu_s_per_iteration"])
                if tian_yau and "schoen" in tian_yau else None,
                "tian_yau_k4": pick((tian_yau or {}).get("tian_yau_k4"), ["solve_s", "iterations", "sigma_final",
                                                                         "reference_record_s"])
                if tian_yau and "tian_yau_k4" in tian_yau else None,
                "p5_10_ensemble": pick((tian_yau or {}).get("p5_10_ensemble"), ["total_s", "reference_total_s",
                                                                               "ty_sigma_final_median"])
                if tian_yau and "p5_10_ensemble" in tian_yau else None,
                "residual_last": residuals[-1], "sigma": sig,
                "sigma_evals_per_s": sigma_per_s, "sigma_evals_per_s_fp64": sigma64_per_s,
                "fp64_iters_per_s": fp64_per_s, "speedup_vs_fp64": (value / fp64_per_s) if fp64_per_s else None,
                "accuracy_vs_fp64": pick(acc, ["h_rel_frobenius", "sigma_rel_err", "sigma_rel_err_same_h",
                                               "iterations"])}
        print(json.dumps(line), flush=True)
    try:
        s.close()
    except Exception:
        if not (serving and "error" in serving):  # a device fault in serving already is in the line
            raise
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
