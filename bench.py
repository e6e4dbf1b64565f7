#!/usr/bin/env python
"""Benchmark of the HCI variational hot path (sparse H build + Davidson) on B200.

Workload (default --config 1): seeded synthetic integrals n = 20 orbitals,
8 alpha + 8 beta electrons, seed 0, HCI threshold eps_var = 5e-5.  The
determinant set is produced, outside the timed region, by this library's own
variational stage on the device (cached under data/).

One timed step is one time-to-E_var solve over that set on the product path:
sparse-H build with FP32 values + FP32 remainder, then Davidson with FP32 sigma
and FP32 basis (FP64 dots, Gram-Schmidt and Rayleigh-Ritz), the learned
preconditioner (DPR fallback), and closing FP64-sigma sweeps, from the
reference's default start until |r| < 1e-4 and |dE| < 1e-8.  The plain FP64
path (FP64 build + the reference's DPR Davidson) is timed beside it on the same
set, and the energy difference of the two is reported (it must stay <= 1 uHa).

Metric: determinants solved per second = N_dets * steps / time (max over ranks),
whole job.  With N GPUs every rank solves its own replica (the single-GPU path
does not shard), so scaling is weak.  Extra keys: both solve times and their
ratio, sigma GB/s against the measured HBM peak, H-build elements/s.
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

METRIC = "time-to-E_var (≤1µHa vs FP64): mixed+learned vs plain GPU; σ GB/s; H elems/s"
CONFIGS = {
    0: dict(n=12, nel=6, eps=1e-4),
    1: dict(n=20, nel=8, eps=5e-5),
    2: dict(n=24, nel=10, eps=2e-5),
    4: dict(n=32, nel=12, eps=1e-5),
}
DAV_MAX_ITER = 2000  # the reference's cap of 50 does not converge on these integrals
# DRAM bytes per algorithmic byte of the upper-triangle FP32 sigma, from one ncu capture
# (config 0 set, 5.82e7 stored pairs: 472.3 MB read + 4.1 MB written for 470 MB); the
# stream grows with the stored pairs, so the ratio carries to larger sets
UPPER_FP32_TRAFFIC_RATIO = 476.4 / 470.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled every 200 ms through NVML in a thread
    (started before the warm-up so that no tool start-up lands in the timed region);
    only samples taken between mark() and stop() are reported."""

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.t_mark = None
        self.running = False

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.hdl = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.hdl, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report it instead of clocks
            self.nv = None
            self.err = str(e)
            return
        self.running = True
        self.t = threading.Thread(target=self._loop, daemon=True)
        self.t.start()

    def _loop(self):
        nv = self.nv
        while self.running:
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.hdl, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.hdl)
                self.samples.append((time.time(), mhz, r))
            except Exception:
                pass
            time.sleep(0.2)

    def mark(self):
        self.t_mark = time.time()

    def stop(self):
        if self.nv is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [f"nvml unavailable: {self.err}"]}
        self.running = False
        self.t.join(timeout=2)
        t1 = time.time()
        nv = self.nv
        names = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                 "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                 "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                 "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        win = [s for s in self.samples if self.t_mark is None or self.t_mark - 0.2 <= s[0] <= t1]
        reasons = sorted({k for _, _, r in win for k, bit in names.items() if r & bit})
        sm = [m for _, m, _ in win]
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(self.max_mhz),
                "reasons": reasons, "samples": len(sm)}


def max_over_ranks(x, world):
    """The largest x over the ranks: a replicated step lasts as long as its slowest rank.
    Every rank calls it at the same point (NCCL reduces on the GPU, gloo on the CPU)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def det_set(cfg_id, device, log=print):
    """The HCI determinant set of a config, made by this library's device variational stage."""
    from risq_b200 import GpuHam, _capi
    from risq_b200.fcidump import synthetic_integrals
    c = CONFIGS[cfg_id]
    ints = synthetic_integrals(c["n"], 0)
    os.makedirs(os.path.join(ROOT, "data"), exist_ok=True)
    path = os.path.join(ROOT, "data", f"hci_n{c['n']}_{c['nel']}_{c['eps']:g}_s0.npz")
    if os.path.exists(path):
        z = np.load(path, allow_pickle=True)
        return ints, z["dets"], z["diag"], float(z["energy"]), list(z["log"])
    t0 = time.time()
    with GpuHam(ints, device) as g:
        # precision -1: FP64 while the matrix fits, FP32 selection solves beyond that
        e, dets, coeffs, diag, vlog = g.variational(c["nel"], c["nel"], c["eps"], max_iter=20,
                                                    dav_max_iter=DAV_MAX_ITER, precision=-1)
    log(f"# det set config {cfg_id}: N={len(dets)} E={e:.10f} ({time.time() - t0:.1f} s)")
    for r in vlog:
        log("#   " + json.dumps({k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()}))
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, dets=dets, diag=diag, coeffs=coeffs, energy=e, log=np.array(vlog, dtype=object))
    os.replace(tmp, path)
    return ints, dets, diag, e, vlog


def cpu_sample(ints, dets, diag, vlog, budget_s=20.0):
    """Oracle (single-threaded C restatement) time-to-E_var on a prefix of the set.

    The HCI list is ordered by selection, so a prefix whose length is one of the
    earlier iterations' sizes is that iteration's variational space; the largest
    such prefix the CPU solves within the budget is used."""
    from oracle import oracle as O
    oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
    sizes = sorted({int(r["n_dets"]) for r in vlog if int(r["n_dets"]) > 2})
    best = None
    for n in sizes:
        t0 = time.perf_counter()
        sp = O.Sparse().build(oh, dets[:n], diag[:n], 0)
        rc, ev, _, st = sp.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER)
        t = time.perf_counter() - t0
        best = dict(n=n, t=t, nnz=sp.nnz, iters=st["iters"], energy=float(ev[0]))
        if t > budget_s / 4:
            break
    return best


def run_reference(args):
    """--impl reference: the CPU path of the reference algorithm on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    ints, dets, diag, e_gpu, vlog = det_set(args.config, 0, log=lambda *a: None)
    times = []
    sample = None
    for i in range(args.warmup + args.steps):
        s = cpu_sample(ints, dets, diag, vlog)
        if i >= args.warmup:
            times.append(s["t"])
            sample = s
    t = float(np.mean(times))
    v = sample["n"] / t
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "dets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"hci n{cfg['n']} {cfg['nel']}a{cfg['nel']}b eps_var {cfg['eps']:g} seed 0",
                   "sample_prefix_dets": sample["n"], "full_dets": int(len(dets))},
        "cpu_baseline": {"value": v, "unit": "dets/s", "cores": 1, "kind": "port",
                         "sample": f"H build + DPR Davidson on the first {sample['n']} of {len(dets)} determinants "
                                   f"(an earlier HCI iteration's space; {sample['nnz']} upper elements, "
                                   f"{sample['iters']} Davidson iterations)"},
        "e2e": {"value": v, "unit": "dets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--impl", default="risq_b200")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--storage", choices=["auto", "upper"], default="auto",
                    help="auto: both triangles when they fit, else the upper triangle; upper: always the "
                         "upper triangle (the reference's SparseMatUpperTri layout)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from risq_b200 import GpuHam, _capi

    def barrier():
        if world > 1:
            dist.barrier()

    def say(*a):
        if rank == 0:
            print(*a, file=sys.stderr, flush=True)

    cfg = CONFIGS[args.config]
    # every rank generates / loads its replica; rank 0 first so the others load the cache
    if rank == 0:
        ints, dets, diag, e_sel, vlog = det_set(args.config, local, log=say)
    barrier()
    if rank != 0:
        ints, dets, diag, e_sel, vlog = det_set(args.config, local, log=lambda *a: None)
    N = len(dets)
    stream = torch.cuda.Stream()
    g = GpuHam(ints, local)
    g.set_stream(stream.cuda_stream)
    ev = lambda: torch.cuda.Event(enable_timing=True)
    from risq_b200 import learned
    model = learned.load_default(ints.norb)
    if model is not None:
        learned.install(g, model)
    precond = _capi.PRECOND_LEARNED if model is not None else _capi.PRECOND_DPR
    g.set_dets(dets, 0, diag)

    def first_fitting(precs):
        for pr in precs:
            try:
                g.build(pr)
                return pr
            except _capi.RisqGpuError as e:
                if e.code != _capi.ERR_OOM:
                    raise
                say(f"# storage {pr} does not fit one GPU")
        raise RuntimeError("no storage mode fits")

    # product path storage: FP32 + FP32 remainder rows when both triangles fit, else the
    # upper triangle (the reference's SparseMatUpperTri layout)
    upper_only = args.storage == "upper"
    precm = first_fitting([_capi.MIXED_UPPER] if upper_only else [_capi.MIXED, _capi.MIXED_UPPER])

    def product_step():
        hs = g.build(precm)
        r = g.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER, mode=_capi.MODE_MIXED, precond=precond)
        return hs, r

    clocks = ClockSampler(local)
    clocks.start()
    for i in range(args.warmup):
        product_step()
    torch.cuda.synchronize()
    barrier()
    clocks.mark()
    t_start, t_end = ev(), ev()
    t_start.record(stream)
    runs = [product_step() for _ in range(args.steps)]
    t_end.record(stream)
    torch.cuda.synchronize()
    ms = t_start.elapsed_time(t_end) / args.steps
    clk = clocks.stop()
    ms_max = max_over_ranks(ms, world)
    barrier()
    hs_m, r_m = runs[-1]
    e_m = float(r_m.eigenvalues[0])

    # kernel launches of one product step, counted by CUPTI (torch.profiler) on an untimed step
    launches_per_step = None
    try:
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            product_step()
            torch.cuda.synchronize()
        launches_per_step = sum(1 for e in prof.events()
                                if e.device_type.name == "CUDA" and e.name.startswith(("k_", "void risq::")))
    except Exception as e:  # profiler unavailable: leave the count out rather than guess
        say(f"# launch count unavailable: {e}")

    # ---- mixed precision with the plain DPR preconditioner (one untimed-loop run) ----
    a, b = ev(), ev()
    torch.cuda.synchronize()
    a.record(stream)
    g.build(precm)
    r_md = g.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER, mode=_capi.MODE_MIXED)
    b.record(stream)
    torch.cuda.synchronize()
    ms_mixed_dpr = a.elapsed_time(b)

    # ---- plain FP64 GPU path on the same set: FP64 build + the reference's DPR Davidson ----
    prec64 = first_fitting([_capi.FP64_UPPER, _capi.COLS] if upper_only else [_capi.FP64, _capi.FP64_UPPER, _capi.COLS])
    plain_ms, plain = [], None
    for i in range(2):
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record(stream)
        hs64 = g.build(prec64)
        r64 = g.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER)
        b.record(stream)
        torch.cuda.synchronize()
        if i > 0:  # the first is a warm-up
            plain_ms.append(a.elapsed_time(b))
        plain = (hs64, r64)
    hs64, r64 = plain
    e64 = float(r64.eigenvalues[0])
    ms_plain = float(np.mean(plain_ms))

    # ---- sigma roofline, FP64 (x, y in the library's internal order) ----
    nnz_u, nnz_f = g.nnz()
    x = torch.randn(N, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    R = 20

    def time_sigma(xx, yy, kind):
        for _ in range(3):
            g.sigma_device(xx.data_ptr(), yy.data_ptr(), kind)
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(R):
            g.sigma_device(xx.data_ptr(), yy.data_ptr(), kind)
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / R

    t_sig = time_sigma(x, y, 0)
    # algorithmic bytes: values (none when recomputed) + int32 columns, per row int64
    # start + int32 length, x and diag read once, y written once; the recomputing
    # kernel also reads both strings of every determinant once (N * 16 B)
    if prec64 == _capi.FP64:
        b_sig = nnz_f * (8 + 4) + N * (8 + 4) + 3 * N * 8
    elif prec64 == _capi.FP64_UPPER:  # each pair once; y is read-modify-written in L2
        b_sig = nnz_u * (8 + 4) + N * (8 + 4) + 3 * N * 8
    else:
        b_sig = nnz_f * 4 + N * (8 + 4) + 3 * N * 8 + N * 16
    peak, peak_kind = peaks()
    sig_gbs = b_sig / (t_sig * 1e-3) / 1e9

    # ---- sigma roofline, FP32 (the product path's dominant kernel) ----
    g.build(precm)
    x32 = x.float()
    y32 = torch.empty_like(x32)
    t_sig32 = time_sigma(x32, y32, 1)
    full_m = precm == _capi.MIXED
    b_sig32 = (nnz_f if full_m else nnz_u) * (4 + 4) + N * (8 + 4) + N * (4 + 4 + 8)
    sig32_gbs = b_sig32 / (t_sig32 * 1e-3) / 1e9

    # ---- end to end through the public API: host dets in, energy + coefficients out ----
    pin = torch.empty((N, 4), dtype=torch.int64, pin_memory=True)
    pin.numpy()[:] = dets.view(np.int64)
    pin_diag = torch.empty(N, dtype=torch.float64, pin_memory=True)
    pin_diag.numpy()[:] = diag
    dets_pinned = pin.numpy().view(np.uint64)
    e2e_ms = []
    for i in range(max(1, min(args.steps, 2))):
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record(stream)
        g.set_dets(dets_pinned, 0, pin_diag.numpy())
        e_api, c_api, _, _ = g.sparse_optimize(None, 1e-4, 1e-8, max_iter=DAV_MAX_ITER, precision=precm,
                                               mode=_capi.MODE_MIXED, precond=precond)
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e = float(np.mean(e2e_ms))
    e2e = max_over_ranks(e2e, world)

    storage = {_capi.FP64: "FP64 both triangles", _capi.FP64_UPPER: "FP64 upper triangle",
               _capi.COLS: "columns only, FP64 elements recomputed in sigma",
               _capi.MIXED: "FP32 + FP32 remainder, both triangles",
               _capi.MIXED_UPPER: "FP32 + FP32 remainder, upper triangle"}
    line = {
        "metric": METRIC,
        "value": N * world / (ms_max * 1e-3),
        "unit": "dets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 sigma / f64 dots, Rayleigh-Ritz and closing sweeps",
        "data": "synthetic",
        "config": {"workload": f"hci n{cfg['n']} {cfg['nel']}a{cfg['nel']}b eps_var {cfg['eps']:g} seed 0",
                   "n_dets": int(N), "nnz_upper": int(nnz_u), "nnz_full": int(nnz_f),
                   "step": "mixed-precision sparse-H build + Davidson (FP32 sigma, learned preconditioner, "
                           "closing FP64 sweeps) to E_var (tol 1e-4, etol 1e-8)",
                   "precond": "learned (MLP, DPR fallback)" if model is not None else "DPR (no network for norb)",
                   "storage": storage[precm], "fp64_storage": storage[prec64],
                   "l2": "CSR stream larger than L2 every step", "parallelism": f"replicas x{world}"},
        "e2e": {"value": N * world / (e2e * 1e-3), "unit": "dets/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": int(N * 40), "d2h_bytes_per_step": int(N * 8 + 8)},
        "roofline": {"bound": "hbm",
                     "kernel": "k_spmv<FP32>" if full_m else "k_spmv_upper<FP32>",
                     "achieved": sig32_gbs, "peak": peak, "unit": "GB/s",
                     "frac": sig32_gbs / peak, "peak_kind": peak_kind,
                     "traffic": None if full_m else int(b_sig32 * UPPER_FP32_TRAFFIC_RATIO),
                     "traffic_source": None if full_m else
                     "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_spmv_upper<float, float> on the "
                     "config 0 set (476.4 MB for 470 MB algorithmic), scaled by the stored pairs",
                     "bytes_per_launch": int(b_sig32), "ms_per_launch": t_sig32},
        "time_to_evar_ms": {"mixed_learned": ms_max, "fp64_plain": ms_plain, "mixed_dpr": ms_mixed_dpr,
                            "mixed_dpr_iters": r_md.stats["iters"],
                            "dE_mixed_dpr_vs_fp64_uHa": abs(float(r_md.eigenvalues[0]) - e64) * 1e6,
                            "speedup_vs_fp64_plain": ms_plain / ms_max,
                            "dE_vs_fp64_uHa": abs(e_m - e64) * 1e6,
                            "mixed_iters": r_m.stats["iters"], "fp64_iters": r64.stats["iters"],
                            "mixed_fp64_sigmas": r_m.stats["n_sigma_fp64"],
                            "learned_fallbacks": r_m.stats["learned_fallbacks"],
                            "mixed_build_ms": hs_m["ms_total"], "fp64_build_ms": hs64["ms_total"]},
        "sigma": {"fp64_kernel": {_capi.FP64: "k_spmv<FP64>", _capi.FP64_UPPER: "k_spmv_upper<FP64>",
                                  _capi.COLS: "k_spmv_otf"}[prec64],
                  "fp64_gbs": sig_gbs, "fp64_ms": t_sig, "fp64_frac": sig_gbs / peak,
                  "fp32_gbs": sig32_gbs, "fp32_ms": t_sig32, "fp32_frac": sig32_gbs / peak},
        "h_build": {"elems_per_s": (nnz_u + N) / (hs64["ms_total"] * 1e-3), "ms": hs64["ms_total"],
                    "gpu_ms_count": hs64["gpu_ms_count"], "gpu_ms_fill": hs64["gpu_ms_fill"],
                    "candidates": hs64["candidates"]},
        "davidson": {"energy_mixed": e_m, "energy_fp64": e64, "e_selection": e_sel,
                     "mixed_ms": r_m.stats["ms_total"], "mixed_ms_sigma": r_m.stats["ms_sigma"],
                     "fp64_ms": r64.stats["ms_total"], "fp64_ms_sigma": r64.stats["ms_sigma"]},
        "clocks": clk,
        "gpu_launches": launches_per_step * args.steps if launches_per_step is not None else None,
        "gpu_launches_per_step": launches_per_step,
    }
    if rank == 0 and not args.no_cpu:
        s = cpu_sample(ints, dets, diag, vlog)
        line["cpu_baseline"] = {"value": s["n"] / s["t"], "unit": "dets/s", "cores": 1, "kind": "port",
                                "sample": f"oracle H build + DPR Davidson on the first {s['n']} of {N} "
                                          f"determinants ({s['nnz']} upper elements, {s['iters']} iterations, "
                                          f"{s['t']:.1f} s)"}
    g.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
