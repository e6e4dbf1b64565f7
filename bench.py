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
path (FP64 build + the reference's DPR Davidson with its 11-vector search
space) is timed beside it on the same set, and the energy difference of the two
is reported (it must stay <= 1 uHa).

Metric: determinants solved per second = N_dets * steps / time (max over ranks),
whole job.  With N GPUs the ranks solve the one set together: each holds a
contiguous share of the row panels of the upper-triangle matrix and every sigma
adds the ranks' 64-bit fixed-point partial sums with an NCCL all-reduce (exact, so
the replicated Davidson solves stay identical); scaling is strong.  Extra keys: the solve times of every leg
and their ratios, sigma GB/s against the measured HBM peak, H-build elements/s,
and a same-set record: the GPU legs and the CPU oracle on the variational space
of an earlier HCI iteration, which the CPU solves in seconds.

--impl reference times the reference's algorithm on the host cores: the CPU
oracle (a C restatement of the reference's Rust path, multi-threaded) runs its
own HCI to that earlier iteration and each step solves that space, so the arm
never loads the GPU library.
"""
from __future__ import annotations

import argparse
import json
import os
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
    # n24: the first 4 HCI iterations (5,042,871 determinants, 5.6e9 upper pairs); the
    # 5th iteration's set (42,294,108 determinants) needs 525 GB for its columns alone,
    # and its matrix-free sigma is timed separately.  Also a 2-root leg.
    2: dict(n=24, nel=10, eps=2e-5, hci_iters=4, two_roots=True),
    4: dict(n=32, nel=12, eps=1e-5),
    # an intermediate set for counter captures (551,147 determinants, a few GB of upper-
    # triangle storage: larger than L2, small enough for a multi-pass ncu capture)
    10: dict(n=20, nel=8, eps=1e-3),
}
DAV_MAX_ITER = 2000  # the reference's cap of 50 does not converge on these integrals
# DRAM bytes (read + write) of one FP32 tiled sigma launch from one ncu capture of the
# kernel on the n20 eps 1e-3 set (profiles/k_sigma_fx_fp32_n20_eps1e-3.md); the
# element stream is the traffic and grows with the stored pairs, so a launch over
# another set is scaled by its pairs
SIGMA32_CAPTURE = {"pairs": 334_413_323, "dram_bytes": 2_696_127_488 + 11_001_088,
                   "set": "n20 8a8b eps_var 1e-3 seed 0 (551,147 dets)"}
# The CPU legs time the variational space of the last HCI iteration whose set holds at
# most this many determinants (the whole set when it is smaller).
CPU_SAMPLE_MAX = 150_000
# Davidson search space of the product path (max_space, keep) for sets of at least
# THICK_MIN_DETS determinants: a thick restart keeping the lowest `keep` Ritz vectors
# (config 1: 107 iterations against the reference space's 197-201).  Below that size a
# Davidson iteration costs as much in launches and the host Rayleigh-Ritz as in sigma,
# and the reference's nroots + 10 with a restart to the Ritz vector (0, 0) is faster
# (config 0: 26 ms against 35 ms for (20, 6)).  The FP32 basis vectors take half the
# memory of FP64 ones.
THICK_SPACE = (32, 8)
THICK_MIN_DETS = 1_000_000
# From this size both paths store the upper triangle in tiles even where both
# triangles would fit: the tiled sigma is the faster one there (n20 eps 1e-3, 551,147
# dets: FP32 0.88 ms against 1.43 ms for both triangles; n24 HCI iteration 4,
# 5,042,871 dets: FP64 27.4 ms against 38.2 ms) and holds half the bytes.
UPPER_MIN_DETS = 500_000


def product_space(n_dets, nroots=1):
    """(max_space, keep) of the product path; (0, 0) is the reference's space
    (nroots + 10, restart to the Ritz vectors)."""
    return THICK_SPACE if n_dets >= THICK_MIN_DETS and THICK_SPACE[1] >= nroots else (0, 0)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_config(cfg_id, world):
    """The `config` dict both arms print (the workload, not how one arm stores it)."""
    c = CONFIGS[cfg_id]
    iters = f", HCI iterations 1-{c['hci_iters']}" if "hci_iters" in c else ""
    return {"workload": f"hci n{c['n']} {c['nel']}a{c['nel']}b eps_var {c['eps']:g} seed 0{iters}",
            "step": "sparse-H build + Davidson to E_var (tol 1e-4, etol 1e-8) from the reference's default start",
            "l2": "CSR stream larger than L2 every step",
            "parallelism": "one GPU" if world == 1 else f"row blocks x{world}, all-reduce of sigma partial sums"}


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


def sum_over_ranks(x, world):
    """The sum of x over the ranks (every rank calls it at the same point)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([int(x)], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t.item())


def det_set(cfg_id, device, log=print):
    """The HCI determinant set of a config, made by this library's device variational stage."""
    from risq_b200 import GpuHam
    from risq_b200.fcidump import synthetic_integrals
    c = CONFIGS[cfg_id]
    ints = synthetic_integrals(c["n"], 0)
    os.makedirs(os.path.join(ROOT, "data"), exist_ok=True)
    max_iter = c.get("hci_iters", 20)
    path = os.path.join(ROOT, "data", f"hci_n{c['n']}_{c['nel']}_{c['eps']:g}_s0_i{max_iter}.npz")
    if os.path.exists(path):
        z = np.load(path, allow_pickle=True)
        return ints, z["dets"], z["diag"], float(z["energy"]), list(z["log"])
    t0 = time.time()
    with GpuHam(ints, device) as g:
        # precision -1: FP64 while the matrix fits, then the upper triangle, then columns only
        e, dets, coeffs, diag, vlog = g.variational(c["nel"], c["nel"], c["eps"], max_iter=max_iter,
                                                    dav_max_iter=DAV_MAX_ITER, precision=-1)
    log(f"# det set config {cfg_id}: N={len(dets)} E={e:.10f} ({time.time() - t0:.1f} s)")
    for r in vlog:
        log("#   " + json.dumps({k: (round(v, 3) if isinstance(v, float) else v) for k, v in r.items()}))
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, dets=dets, diag=diag, coeffs=coeffs, energy=e, log=np.array(vlog, dtype=object))
    os.replace(tmp, path)
    return ints, dets, diag, e, vlog


def sample_iteration(sizes):
    """1-based HCI iteration (and its set size) that the CPU legs time: the last one whose
    set holds at most CPU_SAMPLE_MAX determinants, or the final one."""
    k, n = len(sizes), sizes[-1]
    for i, s in enumerate(sizes):
        if s <= CPU_SAMPLE_MAX:
            k, n = i + 1, s
    return k, n


def oracle_solve(oh, dets, diag):
    """The reference algorithm on every host core: the oracle's fast-rule build and DPR
    Davidson (search space 11, restart to the Ritz vector) from the reference's default
    start.  Returns the time and the result."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    sp = O.Sparse().build_par(oh, dets, diag)
    rc, ev, _, st = sp.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER, parallel=True)
    t = time.perf_counter() - t0
    return dict(t=t, energy=float(ev[0]), iters=st["iters"], nnz=sp.nnz, converged=rc == 0)


def run_reference(args):
    """--impl reference: the reference's algorithm (the CPU oracle, every host core) makes its
    own HCI space and times solves of it; the GPU library is never loaded."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    from risq_b200.fcidump import synthetic_integrals
    cfg = CONFIGS[args.config]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    ints = synthetic_integrals(cfg["n"], 0)
    oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
    # the reference's HCI loop (variational, src/var/mod.rs:59-134) on the host cores, up to the
    # last iteration whose space holds at most CPU_SAMPLE_MAX determinants
    t0 = time.perf_counter()
    hci = O.Hci(oh, cfg["nel"], cfg["nel"], cfg["eps"]).set_options(DAV_MAX_ITER, parallel=True)
    prev = None
    for it in range(cfg.get("hci_iters", 20)):
        rc = hci.step_bounded(CPU_SAMPLE_MAX)
        if rc != 0:
            break
        prev = (it + 1, hci.export())
    if prev is None:
        raise RuntimeError("the first HCI iteration already exceeds the CPU sample bound")
    t_hci = time.perf_counter() - t0
    k, (dets, coeffs, diag) = prev
    n = len(dets)
    times, s = [], None
    for i in range(args.warmup + args.steps):
        s = oracle_solve(oh, dets, diag)
        if i >= args.warmup:
            times.append(s["t"])
    t = float(np.mean(times))
    v = n / t
    threads = O.num_threads()
    out = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "dets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.config, world),
        "cpu_baseline": {"value": v, "unit": "dets/s", "cores": threads, "kind": "port",
                         "sample": f"the variational space of HCI iteration {k} ({n} determinants, {s['nnz']} "
                                   f"upper elements), made by the oracle's own HCI ({t_hci:.0f} s, untimed); "
                                   f"each step builds H and runs DPR Davidson to E_var ({s['iters']} iterations, "
                                   f"E = {s['energy']:.10f})"},
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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle legs")
    ap.add_argument("--sigma-only", action="store_true",
                    help="build the product storage and time `steps` sigma launches (no solve); for counter captures")
    ap.add_argument("--storage", choices=["auto", "upper"], default="auto",
                    help="auto: both triangles when they fit, else the upper triangle; upper: always the "
                         "upper triangle (the reference's SparseMatUpperTri layout, tiled for sigma)")
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
    from risq_b200 import GpuHam, _capi, learned

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
    if world > 1:
        # one set over all ranks: row blocks of the upper triangle, sigma partial sums
        # added by an NCCL all-reduce on the handle's stream
        from risq_b200 import distributed
        g.set_partition(rank, world, distributed.make_allreduce())
    ev = lambda: torch.cuda.Event(enable_timing=True)
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

    def timed(fn):
        a, b = ev(), ev()
        torch.cuda.synchronize()
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), out

    if args.sigma_only:
        prec = _capi.MIXED_UPPER if args.storage == "upper" or world > 1 or N >= UPPER_MIN_DETS else _capi.MIXED
        hs = g.build(prec)
        x32 = torch.randn(N, dtype=torch.float32, device="cuda")
        y32 = torch.empty_like(x32)
        for _ in range(args.warmup):
            g.sigma_device(x32.data_ptr(), y32.data_ptr(), 1)
        ms_s, _ = timed(lambda: [g.sigma_device(x32.data_ptr(), y32.data_ptr(), 1) for _ in range(args.steps)])
        if rank == 0:
            print(json.dumps({"sigma_only": True, "config": workload_config(args.config, world), "n_dets": N,
                              "nnz_upper": hs["nnz_upper"], "n_tiles": hs["n_tiles"], "nnz_dense": hs["nnz_dense"],
                              "fp32_sigma_ms": ms_s / max(args.steps, 1)}))
        barrier()
        g.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # product path storage: FP32 + FP32 remainder rows when both triangles fit, else the
    # upper triangle (the reference's SparseMatUpperTri layout, regrouped into tiles)
    # the partition splits upper-triangle storage
    upper_only = args.storage == "upper" or world > 1 or N >= UPPER_MIN_DETS
    precm = first_fitting([_capi.MIXED_UPPER] if upper_only else [_capi.MIXED, _capi.MIXED_UPPER])

    def solve(prec, mode, pc, space):
        g.set_subspace(*space)
        hs = g.build(prec)
        r = g.davidson(1, None, 1e-4, 1e-8, DAV_MAX_ITER, mode=mode, precond=pc)
        g.set_subspace(0, 0)
        return hs, r

    PRODUCT_SPACE = product_space(N)

    def product_step():
        return solve(precm, _capi.MODE_MIXED, precond, PRODUCT_SPACE)

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

    # ---- other legs on the same set (one run each) ----
    legs = {}
    ms_l, (_, r_l) = timed(lambda: solve(precm, _capi.MODE_MIXED, _capi.PRECOND_DPR, PRODUCT_SPACE))
    legs["mixed_dpr"] = (ms_l, r_l)
    ms_l, (_, r_l) = timed(lambda: solve(precm, _capi.MODE_MIXED, precond, (0, 0)))
    legs["mixed_learned_reference_space"] = (ms_l, r_l)

    # ---- plain FP64 GPU path: FP64 build + the reference's DPR Davidson (11-vector space) ----
    prec64 = first_fitting([_capi.FP64_UPPER, _capi.COLS] if upper_only else [_capi.FP64, _capi.FP64_UPPER, _capi.COLS])
    plain_ms, plain = [], None
    for i in range(2):
        ms_p, out = timed(lambda: solve(prec64, _capi.MODE_FP64, _capi.PRECOND_DPR, (0, 0)))
        if i > 0:  # the first is a warm-up
            plain_ms.append(ms_p)
        plain = out
    hs64, r64 = plain
    e64 = float(r64.eigenvalues[0])
    ms_plain = float(np.mean(plain_ms))
    ms_l, (_, r_l) = timed(lambda: solve(prec64, _capi.MODE_FP64, _capi.PRECOND_DPR, PRODUCT_SPACE))
    legs["fp64_product_space"] = (ms_l, r_l)

    # ---- two roots (block Davidson, davidson.rs:53-79 with nroots = 2): product path
    # against plain FP64, each root within 1 uHa ----
    two_roots = None
    if cfg.get("two_roots"):
        def solve2(prec, mode, pc, space):
            g.set_subspace(*space)
            g.build(prec)
            r = g.davidson(2, None, 1e-4, 1e-8, DAV_MAX_ITER, mode=mode, precond=pc)
            g.set_subspace(0, 0)
            return r
        ms2m, r2m = timed(lambda: solve2(precm, _capi.MODE_MIXED, _capi.PRECOND_DPR, product_space(N, 2)))
        ms2p, r2p = timed(lambda: solve2(prec64, _capi.MODE_FP64, _capi.PRECOND_DPR, (0, 0)))
        two_roots = {"mixed_ms": ms2m, "mixed_iters": r2m.stats["iters"], "mixed_energies": [float(e) for e in r2m.eigenvalues],
                     "fp64_ms": ms2p, "fp64_iters": r2p.stats["iters"], "fp64_energies": [float(e) for e in r2p.eigenvalues],
                     "converged": bool(r2m.converged and r2p.converged),
                     "dE_uHa": [abs(float(a) - float(b)) * 1e6 for a, b in zip(r2m.eigenvalues, r2p.eigenvalues)]}

    # ---- sigma roofline, FP64 (x, y in the library's internal order) ----
    nnz_u, nnz_f = g.nnz()  # this rank's pairs (all of them on one GPU)
    nnz_u_all, nnz_f_all = sum_over_ranks(nnz_u, world), sum_over_ranks(nnz_f, world)
    x = torch.randn(N, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    R = 20

    def time_sigma(xx, yy, kind):
        for _ in range(3):
            g.sigma_device(xx.data_ptr(), yy.data_ptr(), kind)
        ms_s, _ = timed(lambda: [g.sigma_device(xx.data_ptr(), yy.data_ptr(), kind) for _ in range(R)])
        return ms_s / R

    t_sig = time_sigma(x, y, 0)
    tiles64 = int(hs64.get("n_tiles", 0))

    # algorithmic bytes of one sigma: values + int32 column / element index of every stored
    # element, per row its start and length (12 B), x and the diagonal read once, y written
    # once; tiled upper storage also reads 16 B per tile header (20 B for the FP32 sigma,
    # which reads each tile's bound); the recomputing kernel reads both strings of every
    # determinant once (N * 16 B)
    def sigma_bytes(prec, s_v, s_x, n_tiles):
        if prec in (_capi.FP64, _capi.MIXED, _capi.FP32):
            return nnz_f * (s_v + 4) + N * 12 + N * (2 * s_x + 8)
        if prec in (_capi.FP64_UPPER, _capi.MIXED_UPPER, _capi.FP32_UPPER):
            return nnz_u * (s_v + 4) + N * 12 + N * (2 * s_x + 8) + (20 if s_x == 4 else 16) * n_tiles
        return nnz_f * 4 + N * 12 + N * (2 * s_x + 8) + N * 16

    b_sig = sigma_bytes(prec64, 8, 8, tiles64)
    peak, peak_kind = peaks()
    sig_gbs = b_sig / (t_sig * 1e-3) / 1e9

    # ---- sigma roofline, FP32 (the product path's dominant kernel) ----
    hs_p = g.build(precm)
    x32 = x.float()
    y32 = torch.empty_like(x32)
    t_sig32 = time_sigma(x32, y32, 1)
    full_m = precm == _capi.MIXED
    b_sig32 = sigma_bytes(precm, 4, 4, int(hs_p.get("n_tiles", 0)))
    sig32_gbs = b_sig32 / (t_sig32 * 1e-3) / 1e9

    # ---- end to end through the public API: host dets in, energy + coefficients out ----
    pin = torch.empty((N, 4), dtype=torch.int64, pin_memory=True)
    pin.numpy()[:] = dets.view(np.int64)
    pin_diag = torch.empty(N, dtype=torch.float64, pin_memory=True)
    pin_diag.numpy()[:] = diag
    dets_pinned = pin.numpy().view(np.uint64)
    e2e_ms = []
    g.set_subspace(*PRODUCT_SPACE)
    for i in range(max(1, min(args.steps, 2))):
        def api_call():
            g.set_dets(dets_pinned, 0, pin_diag.numpy())
            return g.sparse_optimize(None, 1e-4, 1e-8, max_iter=DAV_MAX_ITER, precision=precm,
                                     mode=_capi.MODE_MIXED, precond=precond)
        ms_e, _ = timed(api_call)
        e2e_ms.append(ms_e)
    g.set_subspace(0, 0)
    e2e = max_over_ranks(float(np.mean(e2e_ms)), world)

    # ---- same set as the CPU sample: an earlier HCI iteration's variational space ----
    sizes = [int(r["n_dets"]) for r in vlog]
    k_s, n_s = sample_iteration(sizes)
    same = None
    cpu = None
    if rank == 0:
        sd, sg = dets[:n_s], diag[:n_s]
        g.set_partition(0, 1)  # the sample is solved by rank 0 alone
        g.set_dets(sd, 0, sg)
        up_s = args.storage == "upper" or n_s >= UPPER_MIN_DETS
        pm_s = _capi.MIXED_UPPER if up_s else _capi.MIXED
        p64_s = _capi.FP64_UPPER if up_s else _capi.FP64
        for _ in range(2):  # warm-up, then timed
            ms_sp, (_, r_sp) = timed(lambda: solve(pm_s, _capi.MODE_MIXED, precond, product_space(n_s)))
            ms_s64, (hs_s64, r_s64) = timed(lambda: solve(p64_s, _capi.MODE_FP64, _capi.PRECOND_DPR, (0, 0)))
        same = {"hci_iteration": k_s, "n_dets": n_s, "nnz_upper": int(hs_s64["nnz_upper"]),
                "gpu_product_ms": ms_sp, "gpu_product_iters": r_sp.stats["iters"],
                "gpu_fp64_plain_ms": ms_s64, "gpu_fp64_iters": r_s64.stats["iters"],
                "e_gpu_fp64": float(r_s64.eigenvalues[0]), "e_gpu_product": float(r_sp.eigenvalues[0])}
        if not args.no_cpu:
            from oracle import oracle as O
            oh = O.Ham.from_arrays(ints.norb, 0, ints.nuc, ints.one_body, ints.two_body)
            cpu = oracle_solve(oh, sd, sg)
            same.update({"cpu_oracle_ms": 1000 * cpu["t"], "cpu_oracle_iters": cpu["iters"],
                         "cpu_threads": O.num_threads(), "e_cpu_oracle": cpu["energy"],
                         "dE_gpu_fp64_vs_oracle_uHa": abs(float(r_s64.eigenvalues[0]) - cpu["energy"]) * 1e6,
                         "nnz_oracle": int(cpu["nnz"]),
                         "ratio_cpu_vs_gpu_product": 1000 * cpu["t"] / ms_sp})

    storage = {_capi.FP64: "FP64 both triangles", _capi.FP64_UPPER: "FP64 upper triangle, tiled",
               _capi.COLS: "columns only, FP64 elements recomputed in sigma",
               _capi.MIXED: "FP32 + FP32 remainder, both triangles",
               _capi.MIXED_UPPER: "FP32 + FP32 remainder, upper triangle, tiled"}
    line = {
        "metric": METRIC,
        "value": N / (ms_max * 1e-3),
        "unit": "dets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32 sigma / f64 dots, Rayleigh-Ritz and closing sweeps",
        "data": "synthetic",
        "config": workload_config(args.config, world),
        "set": {"n_dets": int(N), "nnz_upper": int(nnz_u_all), "nnz_full": int(nnz_f_all),
                "storage": storage[precm], "fp64_storage": storage[prec64],
                "precond": "learned (MLP, DPR fallback)" if model is not None else "DPR (no network for norb)",
                "product_space": {"max_space": PRODUCT_SPACE[0], "keep": PRODUCT_SPACE[1]}},
        "e2e": {"value": N / (e2e * 1e-3), "unit": "dets/s", "ms_per_step": e2e,
                "h2d_bytes_per_step": int(N * 40), "d2h_bytes_per_step": int(N * 8 + 8)},
        "roofline": {"bound": "hbm",
                     "kernel": "k_spmv<FP32>" if full_m else "k_sigma_fx<FP32>",
                     "achieved": sig32_gbs, "peak": peak, "unit": "GB/s",
                     "frac": sig32_gbs / peak, "peak_kind": peak_kind,
                     "traffic": None if full_m else
                     SIGMA32_CAPTURE["dram_bytes"] / SIGMA32_CAPTURE["pairs"] * nnz_u,
                     "traffic_source": None if full_m else
                     f"ncu DRAM bytes of the same kernel on {SIGMA32_CAPTURE['set']}, scaled by stored pairs",
                     "bytes_per_launch": int(b_sig32), "ms_per_launch": t_sig32},
        "time_to_evar_ms": {"mixed_learned": ms_max, "fp64_plain": ms_plain,
                            "speedup_vs_fp64_plain": ms_plain / ms_max,
                            "dE_vs_fp64_uHa": abs(e_m - e64) * 1e6,
                            "mixed_iters": r_m.stats["iters"], "fp64_iters": r64.stats["iters"],
                            "mixed_fp64_sigmas": r_m.stats["n_sigma_fp64"],
                            "learned_fallbacks": r_m.stats["learned_fallbacks"],
                            "mixed_build_ms": hs_m["ms_total"], "fp64_build_ms": hs64["ms_total"],
                            "legs": {k: {"ms": v[0], "iters": v[1].stats["iters"],
                                         "dE_vs_fp64_uHa": abs(float(v[1].eigenvalues[0]) - e64) * 1e6}
                                     for k, v in legs.items()}},
        "sigma": {"fp64_kernel": {_capi.FP64: "k_spmv<FP64>", _capi.FP64_UPPER: "k_sigma_fx<FP64>",
                                  _capi.COLS: "k_spmv_otf"}[prec64],
                  "fp64_gbs": sig_gbs, "fp64_ms": t_sig, "fp64_frac": sig_gbs / peak,
                  "fp32_gbs": sig32_gbs, "fp32_ms": t_sig32, "fp32_frac": sig32_gbs / peak,
                  "tiles": int(hs_p.get("n_tiles", 0)), "pairs_in_dense_tiles": int(hs_p.get("nnz_dense", 0))},
        "h_build": {"elems_per_s": (nnz_u + N) / (hs64["ms_total"] * 1e-3), "ms": hs64["ms_total"],
                    "gpu_ms_count": hs64["gpu_ms_count"], "gpu_ms_fill": hs64["gpu_ms_fill"],
                    "candidates": hs64["candidates"]},
        "davidson": {"energy_mixed": e_m, "energy_fp64": e64, "e_selection": e_sel,
                     "mixed_ms": r_m.stats["ms_total"], "mixed_ms_sigma": r_m.stats["ms_sigma"],
                     "fp64_ms": r64.stats["ms_total"], "fp64_ms_sigma": r64.stats["ms_sigma"]},
        "same_set": same,
        "two_roots": two_roots,
        "clocks": clk,
        "gpu_launches": launches_per_step * args.steps if launches_per_step is not None else None,
        "gpu_launches_per_step": launches_per_step,
    }
    if rank == 0 and cpu is not None:
        # projection of the CPU time to the whole set: the oracle's time per stored pair and
        # Davidson iteration on the sample, times the pairs and iterations of the full solve
        per = cpu["t"] / (max(cpu["nnz"], 1) * max(cpu["iters"], 1))
        proj_s = per * nnz_u_all * r64.stats["iters"]
        line["cpu_baseline"] = {"value": n_s / cpu["t"], "unit": "dets/s", "cores": same["cpu_threads"],
                                "kind": "port",
                                "sample": f"oracle H build + DPR Davidson on the first {n_s} of {N} determinants "
                                          f"(HCI iteration {k_s}; {cpu['nnz']} upper elements, {cpu['iters']} "
                                          f"iterations, {cpu['t']:.1f} s)",
                                "projected_full_set_s": proj_s,
                                "projection": "sample seconds / (sample pairs x sample iterations) x full-set "
                                              "pairs x plain-FP64 GPU iterations on the full set"}
    barrier()
    g.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
