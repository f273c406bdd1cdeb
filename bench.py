"""Benchmark of the fused kNN hot path (GSKNN sgsknn/dgsknn) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one fused-kNN call): the plain sgsknn workload -- N = 1,048,576 float32
points in d = 64 drawn from a 16-Gaussian mixture (sigma 0.05), 65,536 queries and 262,144
references as disjoint seeded index subsets, k = 32, heaps reset to +inf each step. Synthetic,
seeded; the reference publishes no dataset for this path.

`value`  : distance evaluations per second (queries x references / step time) with the point
           table, norms and index lists resident in HBM, through the device entry point.
`e2e`    : the same metric through the reference-facing C ABI (sgsknn_var1) with host buffers:
           each step copies the referenced table rows, norms, index lists and heaps to the GPU
           and the heaps back.
`roofline`: the fused selection kernel's achieved FP32 rate (2d+3 flops per evaluation, the
           reference's count, test/test_dgsknn.c:243) against the CUDA-core FP32 peak at the
           sampled SM clock (148 SMs x 128 lanes x 2 flops x clock).
`cpu_baseline`: the reference's own sgsknn (compiled from its sources, oracle/_ref) on this
           host's cores, on a slice of the queries against all references.

Under torchrun each rank runs an independent replica on its own query set (weak scaling, no
collective on the data path); rank 0 prints one JSON line with the max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS, D_DIM, N_Q, N_R, K_NN = 1 << 20, 64, 65536, 262144, 32
FLOPS_PER_EVAL = 2 * D_DIM + 3
WORKLOAD = (f"plain sgsknn float32: N={N_POINTS} d={D_DIM} gaussian-mixture(16, sigma=0.05), "
            f"queries={N_Q} references={N_R} k={K_NN}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target duration of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--queries", type=int, default=N_Q,
                    help="query count of the device arm (smaller values are for profiling)")
    ap.add_argument("--profile-only", action="store_true",
                    help="device arm only: no end-to-end pass, no CPU baseline, no clocks")
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


# ------------------------------------------------------------------------------------------
# CPU baseline (runs in a child process: its own OpenMP runtime, no CUDA context)
# ------------------------------------------------------------------------------------------
def cpu_worker(spec: str) -> None:
    """Time the reference sgsknn (or the oracle port when the reference library is absent) on
    `q_count` queries against all references. Prints one JSON line."""
    cfg = json.loads(spec)
    nthreads = cfg["threads"]
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    os.environ["GSKNN_IC_NT"] = str(nthreads)
    from rnn_b200 import workloads as W
    p = W.config2(seed=cfg["seed"])
    import ctypes
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libgsknn_ref.so")
    kind = "reference" if os.path.exists(ref_so) else "port"
    if kind == "reference":
        from oracle.oracle import ReferenceLib
        R = ReferenceLib(ref_so)
    else:
        from oracle.oracle import Oracle
        O = Oracle()
        O.set_threads(nthreads)

    def run(qn):
        beta = np.ascontiguousarray(p.beta[:qn])
        D = np.full((qn, p.k), 1.79e30, dtype=np.float32)
        I = np.full((qn, p.k), -1, dtype=np.int32)
        t0 = time.perf_counter()
        if kind == "reference":
            R.var1(p.k, p.X, p.X2, beta, p.X, p.X2, p.alpha, D, I)
        else:
            O.gsknn_ref(p.k, p.X, p.X2, p.alpha, p.X, p.X2, beta, D, I)
        return time.perf_counter() - t0

    # size the sample: at least one MC=104 query block per thread (frame/gsknn.c:975-976)
    q = max(104, min(N_Q, 104 * nthreads // 4))
    t = run(q)
    target = cfg["seconds"]
    while t < target / 4 and q < N_Q:
        q = min(N_Q, int(q * max(2.0, target / max(t, 1e-3) * 0.8)))
        t = run(q)
    out = {"value": q * p.m / t, "seconds": t, "queries": q, "kind": kind, "threads": nthreads}
    print("CPUJSON " + json.dumps(out), flush=True)


def cpu_baseline(seconds: float, threads: int) -> dict:
    spec = json.dumps({"threads": threads, "seconds": seconds, "seed": 2})
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-worker", spec],
                       capture_output=True, text=True, env=env, timeout=600)
    for line in r.stdout.splitlines():
        if line.startswith("CPUJSON "):
            o = json.loads(line[8:])
            return {"value": o["value"], "unit": "distance-evals/s", "cores": o["threads"],
                    "kind": o["kind"],
                    "sample": (f"{o['queries']} of {N_Q} queries x {N_R} references, k={K_NN}, "
                               f"one call, {o['seconds']:.1f} s, GSKNN_IC_NT=OMP_NUM_THREADS="
                               f"{o['threads']}")}
    raise RuntimeError("cpu baseline failed:\n" + r.stdout[-2000:] + r.stderr[-2000:])


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_gpu{gpu_index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# the GPU arm
# ------------------------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import ctypes
    import torch
    from rnn_b200 import gsknn as G
    from rnn_b200 import workloads as W

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    L = G.lib()
    # each rank its own query set (weak scaling); same reference set
    p = W.config2(seed=2)
    nq = args.queries
    if world > 1:
        beta_h = W.permutation(1000 + rank, N_POINTS)[:nq].astype(np.int32)
    else:
        beta_h = np.ascontiguousarray(p.beta[:nq])
    X = torch.from_numpy(p.X).to(dev)
    X2 = torch.from_numpy(p.X2).to(dev)
    alpha = torch.from_numpy(p.alpha).to(dev)
    beta = torch.from_numpy(beta_h).to(dev)
    D = torch.empty((nq, K_NN), dtype=torch.float32, device=dev)
    I = torch.empty((nq, K_NN), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)

    def step():
        D.fill_(float("inf"))
        I.fill_(-1)
        rc = L.gsknn_s_device(N_R, nq, D_DIM, K_NN, X.data_ptr(), X2.data_ptr(), N_POINTS,
                              alpha.data_ptr(), X.data_ptr(), X2.data_ptr(), N_POINTS,
                              beta.data_ptr(), D.data_ptr(), I.data_ptr(), K_NN, st.cuda_stream)
        if rc != 0:
            raise RuntimeError(G.last_error())

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if L.gsknn_stream_status(ctypes.c_void_p(st.cuda_stream)) != 0:
        raise RuntimeError(G.last_error())

    clocks = ClockSampler(local_rank)
    if not args.profile_only:
        clocks.start()
        time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the library brackets each of its kernel launches with CUDA events on its stream
    L.gsknn_trace_read(None, 0)
    L.gsknn_trace_enable(1)
    ev0.record(st)
    for _ in range(args.steps):
        step()
    ev1.record(st)
    torch.cuda.synchronize()
    L.gsknn_trace_enable(0)
    barrier()
    ms = ev0.elapsed_time(ev1) / args.steps
    clk = clocks.stop()
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    trace = read_trace(L)
    launches = sum(v["launches"] for v in trace.values())
    kern = trace.get("fused_knn_simt")
    kern_ms = kern["ms"] / kern["launches"] if kern else None

    evals = float(nq) * N_R
    value = evals * world / (ms * 1e-3)
    if args.profile_only:
        return {"metric": "distance-evals/s", "value": value, "ms_per_step": ms,
                "queries": nq, "kernels": trace, "profile_only": True}

    # end to end through the C ABI with host buffers (sgsknn_var1)
    e2e = e2e_host(L, p, beta_h, args, G)
    out = {
        "metric": "distance-evals/s", "value": value, "unit": "distance-evals/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded gaussian mixture; no dataset published)",
        "mode": "plain FP32 CUDA-core fused kernel",
        "config": {"workload": WORKLOAD, "points": N_POINTS, "d": D_DIM, "queries": N_Q,
                   "references": N_R, "k": K_NN, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (256 MiB point table gathered every step)"},
        "gpu_launches": launches,
        "kernels": trace,
        "clocks": clk,
    }
    if kern_ms is not None:
        sm_mhz = clk.get("sm_mhz") or 1965.0
        peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
        achieved = evals * FLOPS_PER_EVAL / (kern_ms * 1e-3) / 1e12
        out["roofline"] = {"bound": "fp32-cuda-core", "achieved": achieved, "peak": peak,
                           "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                           "kernel": "fused_knn_simt", "kernel_ms": kern_ms,
                           "peak_source": "nominal FP32 issue rate at the sampled SM clock"}
    out["e2e"] = e2e
    return out


def read_trace(L) -> dict:
    """Per-kernel launch counts and total milliseconds recorded by the library's tracer."""
    import ctypes
    buf = ctypes.create_string_buffer(1 << 16)
    L.gsknn_trace_read(buf, ctypes.c_int(len(buf)))
    return json.loads(buf.value.decode() or "{}")


def e2e_host(L, p, beta_h, args, G):
    import ctypes
    import torch
    Xh, X2h = p.X, p.X2
    alpha_h = p.alpha
    D = np.empty((N_Q, K_NN), dtype=np.float32)
    I = np.empty((N_Q, K_NN), dtype=np.int32)
    c_i = ctypes.c_int

    def call():
        D.fill(np.inf)
        I.fill(-1)
        L.sgsknn_var1(c_i(N_Q), c_i(N_R), c_i(D_DIM), c_i(K_NN), G._p(Xh), G._p(X2h),
                      G._p(beta_h), G._p(Xh), G._p(X2h), G._p(alpha_h), G._p(D), G._p(I))
        code, msg = G.last_error()
        if code != 0:
            raise RuntimeError(msg)

    call()
    steps = max(2, min(args.steps, 5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        call()
    t = (time.perf_counter() - t0) / steps
    lo = int(min(beta_h.min(), alpha_h.min()))
    hi = int(max(beta_h.max(), alpha_h.max()))
    rows = hi - lo + 1
    h2d = rows * D_DIM * 4 + rows * 4 + (N_Q + N_R) * 4 + 2 * N_Q * K_NN * 4
    d2h = 2 * N_Q * K_NN * 4
    return {"value": float(N_Q) * N_R / t, "unit": "distance-evals/s", "ms_per_step": t * 1e3,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": "sgsknn_var1 (host pointers, pageable numpy buffers)"}


def main():
    args = parse()
    if args.cpu_worker:
        cpu_worker(args.cpu_worker)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    if args.impl == "reference":
        # the reference's CPU implementation of the path; rank 0 alone
        if rank != 0:
            return
        cb = cpu_baseline(max(5.0, args.cpu_seconds), threads)
        out = {"impl": "reference", "metric": "distance-evals/s", "value": cb["value"],
               "unit": "distance-evals/s", "n_gpus": args.gpus, "steps": args.steps,
               "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded gaussian mixture)",
               "config": {"workload": WORKLOAD, "points": N_POINTS, "d": D_DIM, "queries": N_Q,
                          "references": N_R, "k": K_NN},
               "cpu_baseline": cb,
               "e2e": {"value": cb["value"], "unit": "distance-evals/s",
                       "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
        return

    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    out = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile_only:
        try:
            out["cpu_baseline"] = cpu_baseline(args.cpu_seconds, threads)
        except Exception as e:  # reported, not fatal
            out["cpu_baseline"] = {"error": str(e)[-400:]}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
