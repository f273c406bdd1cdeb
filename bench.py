"""Benchmark of the fused kNN hot path (GSKNN sgsknn/dgsknn) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one fused-kNN call): the plain sgsknn workload -- N = 1,048,576 float32
points in d = 64 drawn from a 16-Gaussian mixture (sigma 0.05), 65,536 queries and 262,144
references as disjoint seeded index subsets, k = 32, heaps reset to +inf each step. Synthetic,
seeded; the reference publishes no dataset for this path.

`value`  : distance evaluations per second (queries x references / step time) with the point
           table, norms and index lists resident in HBM, through the device entry point, in
           the library's default arithmetic (AUTO: tensor-core distances + FP64 re-rank, which
           returns the exact FP64 neighbour sets).
`e2e`    : the same metric through the reference-facing C ABI (sgsknn_var1) with host buffers:
           each step copies the referenced table rows, norms, index lists and heaps to the GPU
           and the heaps back.
`modes`  : the same workload per arithmetic: plain FP32 CUDA-core kernel, TF32, BF16 and split
           BF16 tensor-core forms.
`precision_form`: the precision workload (32,768 queries x 262,144 references, d = 256, k = 64,
           points on an 8-dim latent manifold + noise): TF32 / BF16 tensor-core + FP64 re-rank
           against the plain FP32 kernel, with the tensor pipe's roofline.
`batching_form`: all-nearest-neighbour search over randomized-tree leaves (N = 2,097,152 points
           of the same kind of mixture, d = 64, k = 32, 8 trees per pass, leaves of 256..2048
           points, alpha = beta = leaf, 4 passes merged into one heap): every leaf of a pass in
           one persistent launch replayed from a CUDA graph, tile shape by the autotuner;
           distance evaluations (sum of leaf sizes squared) per second over the 4 passes.
           `streaming`: the same passes with the point table and heaps in host memory,
           streamed through the device in groups of 524,288 points (the form for point sets
           beyond HBM).
`serving_form`: requests against a resident reference set (4,194,304 points, d = 128,
           U[0,1)): Poisson arrivals, m log-uniform in [1, 4096] queries, k from {8, 16, 64};
           continuous batching inside the library; p50 / p99 latency (submit to result on the
           device) and aggregate distance evaluations/s, beside the same requests run one by
           one through the plain FP32 kernel and through the per-call tensor-core path.
`roofline`: the dominant kernel of the headline run; contraction counted as 2d flops per
           evaluation, against the measured bf16 dense peak (MEASURED_PEAKS.json; half of it
           for TF32, the TF32 tensor rate) or, for the CUDA-core kernel, the FP32 issue rate at
           the sampled SM clock.
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
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS, D_DIM, N_Q, N_R, K_NN = 1 << 20, 64, 65536, 262144, 32
WORKLOAD = (f"plain sgsknn float32: N={N_POINTS} d={D_DIM} gaussian-mixture(16, sigma=0.05), "
            f"queries={N_Q} references={N_R} k={K_NN}")
MODE_NAMES = {0: "auto", 1: "fp32", 2: "tf32", 3: "bf16", 4: "bf16x3"}
DOMINANT = {"fp32": "fused_knn_simt", "tf32": "tc_knn", "bf16": "tc_knn", "bf16x3": "tc_knn"}


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
    ap.add_argument("--mode", default="auto", choices=list(MODE_NAMES.values()),
                    help="arithmetic of the headline run")
    ap.add_argument("--profile-only", action="store_true",
                    help="headline device run only: no e2e, modes, precision form, CPU baseline")
    ap.add_argument("--precision-only", action="store_true",
                    help="only the precision-form workload (d=256), for profiling")
    ap.add_argument("--pf-modes", default="fp32,tf32,bf16,bf16x3",
                    help="modes of the precision-form workload")
    ap.add_argument("--pf-queries", type=int, default=32768,
                    help="query count of the precision-form workload (smaller for profiling)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching-form workload")
    ap.add_argument("--batch-only", action="store_true",
                    help="only the batching-form workload (all-NN over tree leaves)")
    ap.add_argument("--batch-points", type=int, default=1 << 21,
                    help="points of the batching-form workload (smaller for profiling)")
    ap.add_argument("--batch-passes", type=int, default=4)
    ap.add_argument("--stream-group", type=int, default=1 << 19,
                    help="points per group of the streaming measurement (0: skip it)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-form workload")
    ap.add_argument("--serve-only", action="store_true",
                    help="only the serving-form workload (Poisson requests, resident set)")
    ap.add_argument("--serve-refs", type=int, default=1 << 22,
                    help="resident reference points of the serving workload")
    ap.add_argument("--serve-requests", type=int, default=400)
    ap.add_argument("--serve-slice", type=int, default=0,
                    help="rows per serving batch (0: the engine's default, ~3 ms of work)")
    ap.add_argument("--serve-slots", type=int, default=2, help="serving stream slots")
    ap.add_argument("--serve-mode", default="auto", choices=list(MODE_NAMES.values()),
                    help="arithmetic of the serving engine (a tensor-core mode or auto)")
    ap.add_argument("--serve-rate", type=float, default=150.0,
                    help="mean request arrival rate (requests/s, Poisson)")
    ap.add_argument("--kernel-case", default=None,
                    choices=["config1", "large_k", "tc_q8192", "batch_small", "serve_one",
                             "fp32_q8192", "batch_small_tc"],
                    help="one small run of one path, for per-kernel profiling: warm-up call, "
                         "then the profiled call")
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "bf16": d.get("bf16_tflops", 1590.0),
                "bf16_sustained": d.get("bf16_tflops_sustained", 1400.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0, "source": "fallback"}


# ------------------------------------------------------------------------------------------
# CPU baseline (runs in a child process: its own OpenMP runtime, no CUDA context)
# ------------------------------------------------------------------------------------------
def cpu_worker(spec: str) -> None:
    """Time the reference sgsknn (or the oracle port when the reference library is absent) on
    a slice of the queries against all references. Prints one JSON line."""
    cfg = json.loads(spec)
    nthreads = cfg["threads"]
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    os.environ["GSKNN_IC_NT"] = str(nthreads)
    from rnn_b200 import workloads as W
    if cfg.get("kind") == "batch":
        batch_cpu_worker(cfg, nthreads)
        return
    if cfg.get("kind") == "config1":
        config1_cpu_worker(cfg, nthreads)
        return
    if cfg.get("kind") in ("config3", "config5"):
        slice_cpu_worker(cfg, nthreads)
        return
    p = W.config2(seed=cfg["seed"])
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

    # size the sample: at least one MC=104 query block per thread, since the reference spreads
    # its query blocks over the threads (frame/gsknn.c:975-976)
    q = max(104, min(N_Q, 104 * nthreads))
    t = run(q)
    target = cfg["seconds"]
    while t < target / 4 and q < N_Q:
        q = min(N_Q, int(q * max(2.0, target / max(t, 1e-3) * 0.8)))
        t = run(q)
    steps, warmup = cfg.get("steps", 1), cfg.get("warmup", 0)
    times = [t]
    if steps > 1 or warmup > 0:  # the sizing call is the first warm-up; then W more, K timed
        for _ in range(max(0, warmup - 1)):
            run(q)
        times = [run(q) for _ in range(steps)]
    t = sum(times)
    out = {"value": q * p.m * len(times) / t, "seconds": t, "queries": q, "kind": kind,
           "threads": nthreads, "steps": len(times), "ms_per_step": 1e3 * t / len(times)}
    print("CPUJSON " + json.dumps(out), flush=True)


def batch_cpu_worker(cfg, nthreads) -> None:
    """The reference's sgsknn once per leaf (alpha = beta = leaf), as its tree drivers run it,
    over the leaves of one tree of the batching workload until the time target is reached."""
    from rnn_b200 import batch as B
    from rnn_b200 import workloads as W
    from oracle.oracle import ReferenceLib
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libgsknn_ref.so")
    p = W.config4(seed=cfg["seed"], n_points=cfg["points"])
    lv = B.rkdt_leaves(p.X, 1, p.leaf_min, p.leaf_max, seed=p.tree_seed)
    R = ReferenceLib(ref_so)
    evals, t, n = 0.0, 0.0, 0
    for l in range(lv.nleaves):
        leaf = np.ascontiguousarray(lv.pts[lv.ptr[l]:lv.ptr[l + 1]])
        D = np.full((leaf.size, p.k), 1.79e30, dtype=np.float32)
        I = np.full((leaf.size, p.k), -1, dtype=np.int32)
        t0 = time.perf_counter()
        R.var1(p.k, p.X, p.X2, leaf, p.X, p.X2, leaf, D, I)
        t += time.perf_counter() - t0
        evals += float(leaf.size) ** 2
        n += 1
        if t >= cfg["seconds"]:
            break
    print("CPUJSON " + json.dumps({"value": evals / t, "seconds": t, "leaves": n,
                                   "kind": "reference", "threads": nthreads}), flush=True)


def config1_cpu_worker(cfg, nthreads) -> None:
    """The reference's dgsknn (its AVX double path, frame/gsknn.c:1138-1184) on the config-1
    workload: one step = two merging calls into a heapCreate_d heap, as the GPU leg runs it."""
    from rnn_b200 import workloads as W
    from oracle.oracle import ReferenceLib
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libgsknn_ref.so")
    p, alpha2 = W.config1(1)
    R = ReferenceLib(ref_so)

    def step():
        h = R.heap_create(p.n, p.k, 1.79e308, double=True)
        t0 = time.perf_counter()
        R.gsknn(p.k, p.X, p.X2, p.alpha, p.X, p.X2, p.beta, h)
        R.gsknn(p.k, p.X, p.X2, alpha2, p.X, p.X2, p.beta, h)
        t = time.perf_counter() - t0
        R.heap_free(h, double=True)
        return t

    for _ in range(2):
        step()
    times = []
    while sum(times) < cfg["seconds"] and len(times) < 200:
        times.append(step())
    t = sum(times) / len(times)
    print("CPUJSON " + json.dumps({"value": 2.0 * p.n * p.m / t, "ms_per_step": 1e3 * t,
                                   "steps": len(times), "kind": "reference",
                                   "threads": nthreads}), flush=True)


def slice_cpu_worker(cfg, nthreads) -> None:
    """The reference's sgsknn_var1 on a query slice of the precision-form workload (config 3:
    262,144 latent-manifold references, d = 256, k = 64) or of the serving workload (config 5:
    4,194,304 resident U[0,1) references, d = 128, k = 64): one block of 104 queries per thread
    (the reference spreads its query blocks over the threads), one call."""
    from rnn_b200 import workloads as W
    from oracle.oracle import ReferenceLib
    ref_so = os.path.join(ROOT, "oracle", "_ref", "libgsknn_ref.so")
    R = ReferenceLib(ref_so)
    q = 104 * nthreads
    if cfg["kind"] == "config3":
        p = W.config3(seed=3)
        X, X2, alpha, k = p.X, p.X2, p.alpha, p.k
        beta = np.ascontiguousarray(p.beta[:q])
    else:
        nref, d, k = 1 << 22, 128, 64
        X = np.empty((nref + q, d), dtype=np.float32)
        X[:nref] = W.uniform_table(71, nref, d, np.float32)
        X[nref:] = W.uniform_table(72, q, d, np.float32)
        X2 = W.sq_norms(X)
        alpha = np.arange(nref, dtype=np.int32)
        beta = np.arange(nref, nref + q, dtype=np.int32)
    D = np.full((q, k), 1.79e30, dtype=np.float32)
    I = np.full((q, k), -1, dtype=np.int32)
    t0 = time.perf_counter()
    R.var1(k, X, X2, beta, X, X2, alpha, D, I)
    t = time.perf_counter() - t0
    print("CPUJSON " + json.dumps({"value": float(q) * alpha.size / t, "seconds": t,
                                   "queries": q, "references": int(alpha.size), "k": k,
                                   "kind": "reference", "threads": nthreads}), flush=True)


def slice_cpu_baseline(kind: str, threads: int) -> dict:
    spec = json.dumps({"kind": kind, "threads": threads})
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-worker", spec],
                       capture_output=True, text=True, env=env, timeout=900)
    for line in r.stdout.splitlines():
        if line.startswith("CPUJSON "):
            o = json.loads(line[8:])
            return {"value": o["value"], "unit": "distance-evals/s", "cores": o["threads"],
                    "kind": o["kind"],
                    "sample": (f"reference sgsknn_var1, {o['queries']} queries x "
                               f"{o['references']} references, k={o['k']}, one call, "
                               f"{o['seconds']:.1f} s, GSKNN_IC_NT=OMP_NUM_THREADS="
                               f"{o['threads']}")}
    raise RuntimeError(kind + " cpu baseline failed:\n" + r.stdout[-2000:] + r.stderr[-2000:])


def config1_cpu_baseline(seconds: float, threads: int) -> dict:
    spec = json.dumps({"kind": "config1", "threads": threads, "seconds": seconds})
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-worker", spec],
                       capture_output=True, text=True, env=env, timeout=600)
    for line in r.stdout.splitlines():
        if line.startswith("CPUJSON "):
            o = json.loads(line[8:])
            return {"value": o["value"], "unit": "distance-evals/s", "cores": o["threads"],
                    "kind": o["kind"], "ms_per_step": o["ms_per_step"],
                    "sample": (f"reference dgsknn, two merging calls per step into a "
                               f"heapCreate_d heap, {o['steps']} steps, "
                               f"GSKNN_IC_NT=OMP_NUM_THREADS={o['threads']}")}
    raise RuntimeError("config-1 cpu baseline failed:\n" + r.stdout[-2000:] + r.stderr[-2000:])


def batch_cpu_baseline(seconds: float, threads: int, points: int) -> dict:
    spec = json.dumps({"kind": "batch", "threads": threads, "seconds": seconds, "seed": 4,
                       "points": points})
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-worker", spec],
                       capture_output=True, text=True, env=env, timeout=900)
    for line in r.stdout.splitlines():
        if line.startswith("CPUJSON "):
            o = json.loads(line[8:])
            return {"value": o["value"], "unit": "distance-evals/s", "cores": o["threads"],
                    "kind": o["kind"],
                    "sample": (f"reference sgsknn_var1 per leaf (alpha = beta = leaf), "
                               f"{o['leaves']} leaves of one tree, {o['seconds']:.1f} s, "
                               f"GSKNN_IC_NT=OMP_NUM_THREADS={o['threads']}")}
    raise RuntimeError("batch cpu baseline failed:\n" + r.stdout[-2000:] + r.stderr[-2000:])


def cpu_baseline(seconds: float, threads: int, steps: int = 1, warmup: int = 0) -> dict:
    """The reference sgsknn on the host cores: a query slice against all references, sized to
    about `seconds` per call; with steps/warmup, `warmup` untimed calls then `steps` timed ones."""
    spec = json.dumps({"threads": threads, "seconds": seconds, "seed": 2, "steps": steps,
                       "warmup": warmup})
    env = dict(os.environ)
    env["CUDA_VISIBLE_DEVICES"] = ""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--cpu-worker", spec],
                       capture_output=True, text=True, env=env, timeout=600)
    for line in r.stdout.splitlines():
        if line.startswith("CPUJSON "):
            o = json.loads(line[8:])
            calls = "one call" if o["steps"] == 1 else f"{o['steps']} timed calls"
            return {"value": o["value"], "unit": "distance-evals/s", "cores": o["threads"],
                    "kind": o["kind"], "ms_per_step": o["ms_per_step"],
                    "sample": (f"{o['queries']} of {N_Q} queries x {N_R} references, k={K_NN}, "
                               f"{calls}, {o['seconds']:.1f} s, GSKNN_IC_NT=OMP_NUM_THREADS="
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
        fd, self.path = tempfile.mkstemp(prefix=f"gsknn_clocks_gpu{gpu_index}_", suffix=".csv")
        os.close(fd)

    def start(self):
        try:
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
        try:
            os.unlink(self.path)
        except OSError:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": ["unsampled"]}
        loaded = [s for s in sm if s > 0.5 * max(sm)] or sm
        return {"sm_mhz": float(np.median(loaded)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# the GPU arm
# ------------------------------------------------------------------------------------------
def read_trace(L) -> dict:
    """Per-kernel launch counts and total milliseconds recorded by the library's tracer."""
    import ctypes
    buf = ctypes.create_string_buffer(1 << 16)
    L.gsknn_trace_read(buf, ctypes.c_int(len(buf)))
    return json.loads(buf.value.decode() or "{}")


class DeviceProblem:
    """A float kNN problem resident on the device, callable through gsknn_s_device."""

    def __init__(self, p, beta_h, dev):
        import torch
        self.torch = torch
        self.p = p
        self.nq = beta_h.size
        self.X = torch.from_numpy(p.X).to(dev)
        self.X2 = torch.from_numpy(p.X2).to(dev)
        self.alpha = torch.from_numpy(p.alpha).to(dev)
        self.beta = torch.from_numpy(beta_h).to(dev)
        self.D = torch.empty((self.nq, p.k), dtype=torch.float32, device=dev)
        self.I = torch.empty((self.nq, p.k), dtype=torch.int32, device=dev)
        self.st = torch.cuda.current_stream(dev)

    @property
    def evals(self):
        return float(self.nq) * self.p.m

    def step(self, L, G):
        self.D.fill_(float("inf"))
        self.I.fill_(-1)
        n_rows = self.p.X.shape[0]
        rc = L.gsknn_s_device(self.p.m, self.nq, self.p.d, self.p.k, self.X.data_ptr(),
                              self.X2.data_ptr(), n_rows, self.alpha.data_ptr(),
                              self.X.data_ptr(), self.X2.data_ptr(), n_rows,
                              self.beta.data_ptr(), self.D.data_ptr(), self.I.data_ptr(),
                              self.p.k, self.st.cuda_stream)
        if rc != 0:
            raise RuntimeError(G.last_error())


def timed(L, G, prob, mode, steps, warmup, barrier=None, clocks=None):
    """Warm-up, then `steps` calls bracketed by events on the launching stream with the
    library's per-kernel tracer on. Returns (ms per step, trace)."""
    import ctypes
    torch = prob.torch
    G.set_mode(mode)
    for _ in range(warmup):
        prob.step(L, G)
    torch.cuda.synchronize()
    if L.gsknn_stream_status(ctypes.c_void_p(prob.st.cuda_stream)) != 0:
        raise RuntimeError(G.last_error())
    if clocks:
        clocks.start()
        time.sleep(0.3)
    if barrier:
        barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    read_trace(L)
    L.gsknn_trace_enable(1)
    ev0.record(prob.st)
    for _ in range(steps):
        prob.step(L, G)
    ev1.record(prob.st)
    torch.cuda.synchronize()
    L.gsknn_trace_enable(0)
    if barrier:
        barrier()
    if L.gsknn_stream_status(ctypes.c_void_p(prob.st.cuda_stream)) != 0:
        raise RuntimeError(G.last_error())
    return ev0.elapsed_time(ev1) / steps, read_trace(L)


# DRAM bytes per launch of the dominant kernel, from one ncu capture of this same workload
# (dram__bytes_read.sum + dram__bytes_write.sum; profiles/launch_list_headline_config2.md)
TRAFFIC = {("tc_knn", "bf16x3", N_Q): 280260352 + 315675136}


def roofline(mode_name, prob, trace, peaks, clk):
    kname = DOMINANT[mode_name]
    kern = trace.get(kname)
    if not kern:
        return None
    kms = kern["ms"] / kern["launches"]
    d = prob.p.d
    if mode_name == "fp32":
        flops = prob.evals * (2 * d + 3)
        sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
        peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
        src = "nominal FP32 CUDA-core issue rate at the sampled SM clock"
        bound = "fp32"
    else:
        flops = prob.evals * 2 * d
        if mode_name == "tf32" and peaks.get("tf32_tflops"):
            peak = peaks["tf32_tflops"]
            src = "measured TF32 dense GEMM burst rate (peak_probes)"
        else:
            peak = peaks["bf16"] * (0.5 if mode_name == "tf32" else 1.0)
            src = (f"{peaks['source']} bf16 dense burst peak"
                   + (" x 0.5 (TF32 tensor rate, not probed)" if mode_name == "tf32" else ""))
        bound = "tensor"
    achieved = flops / (kms * 1e-3) / 1e12
    out = {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
           "frac": achieved / peak, "traffic": TRAFFIC.get((kname, mode_name, prob.nq)),
           "kernel": kname, "kernel_ms": kms, "peak_source": src}
    if mode_name == "bf16x3":
        out["executed_frac"] = 3 * achieved / peak
        out["note"] = "split BF16 runs 3 MMAs per product; achieved counts the 2d useful flops"
    return out



# ------------------------------------------------------------------------------------------
# measured rates that MEASURED_PEAKS.json does not carry
# ------------------------------------------------------------------------------------------
def _gemm_tflops(torch, a, b, reps=5):
    for _ in range(3):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) * 1e-3
        best = t if best is None else min(best, t)
    n = a.shape[0]
    return 2.0 * n * a.shape[1] * b.shape[1] / best / 1e12


def peak_probes(dev) -> dict:
    """Dense GEMM rates measured on this GPU through cuBLAS (torch.matmul), each timed alone,
    best of 5 after warm-up: TF32 (float32 operands with TF32 tensor math, 8192^3) and FP64
    (4096^3). They are the denominators of the TF32 and FP64 rooflines."""
    import torch
    out = {}
    prev = torch.backends.cuda.matmul.allow_tf32
    try:
        torch.backends.cuda.matmul.allow_tf32 = True
        a = torch.randn(8192, 8192, device=dev)
        b = torch.randn(8192, 8192, device=dev)
        out["tf32_tflops"] = _gemm_tflops(torch, a, b)
        del a, b
        a = torch.randn(4096, 4096, device=dev, dtype=torch.float64)
        b = torch.randn(4096, 4096, device=dev, dtype=torch.float64)
        out["fp64_tflops"] = _gemm_tflops(torch, a, b)
        del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
        torch.cuda.empty_cache()
    out["how"] = ("torch.matmul burst, best of 5 (CUDA events): float32 8192^3 with TF32 "
                  "tensor math; float64 4096^3")
    return out


# ------------------------------------------------------------------------------------------
# accuracy of a result against FP64 (computed here with torch in float64 on the GPU)
# ------------------------------------------------------------------------------------------
def accuracy(L, G, X, X2, alpha, beta, D, I, mode_name, nsample=256, seed=17):
    """On `nsample` seeded rows: the FP64 distances of the returned ids (float inputs upcast,
    the caller's norms, (-2<q,c> + |c|^2) + |q|^2 clamped at 0) against the returned values
    (max relative error), and whether they equal the k smallest FP64 distances of the row over
    all candidates (exact recall, tie-robust). For tensor-core modes also max |d' - d| / E of
    the approximate distances of `nsample` rows against all candidates."""
    import ctypes
    import torch
    from rnn_b200 import workloads as W
    n, k = D.shape
    rows = torch.from_numpy(np.sort(W.permutation(seed, n)[:nsample]).astype(np.int64)).to(
        D.device)
    q = beta[rows].long()
    Xq = X[q].double()
    qq = X2[q].double()
    Xc = X[alpha.long()].double()
    cc = X2[alpha.long()].double()
    full = torch.clamp(-2.0 * Xq @ Xc.T + cc[None, :] + qq[:, None], min=0.0)
    best = torch.topk(full, k, dim=1, largest=False, sorted=True).values
    ids = I[rows].long()
    ok = ids >= 0
    # FP64 distance of each returned id, read from the same block (position of the id in the
    # candidate list; a repeated id has one distance)
    pos = torch.full((X.shape[0],), -1, dtype=torch.long, device=D.device)
    pos[alpha.long()] = torch.arange(alpha.numel(), device=D.device)
    pid = pos[ids.clamp(min=0)]
    ok = ok & (pid >= 0)
    got = torch.where(ok, full.gather(1, pid.clamp(min=0)), torch.full_like(best, float("inf")))
    rel = ((D[rows].double() - got).abs() / got.clamp(min=1e-30))[ok]
    exact_rows = int((torch.sort(got, dim=1).values == best).all(dim=1).sum().item())
    res = {"rows_checked": int(nsample), "rows_exact_fp64_recall": exact_rows,
           "max_rel_dist_err": float(rel.max().item()) if rel.numel() else 0.0}
    del full
    tc = {"tf32": 2, "bf16": 3, "bf16x3": 4}.get(mode_name)
    if tc is not None:
        f = L.gsknn_tc_distances
        vp, ci, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        f.argtypes = [ci, ci, ci, ci, ci, vp, vp, ll, vp, vp, vp, ll, vp, vp, vp, ci, vp, ll,
                      vp, vp]
        f.restype = ci
        m, d = alpha.numel(), X.shape[1]
        sub = beta[rows].contiguous()
        Dd = torch.full((nsample, k), float("inf"), device=D.device)
        Id = torch.full((nsample, k), -1, dtype=torch.int32, device=D.device)
        C = torch.empty((nsample, m), device=D.device)
        margin = torch.zeros(nsample, device=D.device)
        st = torch.cuda.current_stream(D.device)
        rc = f(tc, m, nsample, d, k, X.data_ptr(), X2.data_ptr(), X.shape[0], alpha.data_ptr(),
               X.data_ptr(), X2.data_ptr(), X.shape[0], sub.data_ptr(), Dd.data_ptr(),
               Id.data_ptr(), k, C.data_ptr(), m, margin.data_ptr(), st.cuda_stream)
        torch.cuda.synchronize()
        if rc == 0:
            exu = -2.0 * Xq @ Xc.T + cc[None, :] + qq[:, None]
            E = margin.double()[:, None] / 2.0
            res["max_err_over_E"] = float(((C.double() - exu).abs() / E).max().item())
            res["median_E"] = float(E.median().item())
            del exu
        del C
    torch.cuda.empty_cache()
    return res


# ------------------------------------------------------------------------------------------
# config 1: plain dgsknn, FP64
# ------------------------------------------------------------------------------------------
def fp64_config1(L, G, W, dev, peaks, args):
    """dgsknn in float64: N=8192, d=32, U[0,1), 4096 queries, 4096 candidates, k=16; one step =
    two calls, the second with a fresh candidate list merging into the same heaps."""
    import ctypes
    import torch
    p, alpha2 = W.config1(1)
    X = torch.from_numpy(p.X).to(dev)
    X2 = torch.from_numpy(p.X2).to(dev)
    a1 = torch.from_numpy(p.alpha).to(dev)
    a2 = torch.from_numpy(alpha2).to(dev)
    b = torch.from_numpy(p.beta).to(dev)
    D = torch.empty((p.n, p.k), dtype=torch.float64, device=dev)
    I = torch.empty((p.n, p.k), dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    N = p.X.shape[0]

    def step():
        D.fill_(float("inf"))
        I.fill_(-1)
        for a in (a1, a2):
            rc = L.gsknn_d_device(p.m, p.n, p.d, p.k, X.data_ptr(), X2.data_ptr(), N,
                                  a.data_ptr(), X.data_ptr(), X2.data_ptr(), N, b.data_ptr(),
                                  D.data_ptr(), I.data_ptr(), p.k, st.cuda_stream)
            if rc != 0:
                raise RuntimeError(G.last_error())

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    steps = max(20, args.steps)
    read_trace(L)
    L.gsknn_trace_enable(1)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        step()
    e1.record(st)
    torch.cuda.synchronize()
    L.gsknn_trace_enable(0)
    tr = read_trace(L)
    ms = e0.elapsed_time(e1) / steps
    evals = 2.0 * p.n * p.m
    if L.gsknn_stream_status(ctypes.c_void_p(st.cuda_stream)) != 0:
        raise RuntimeError(G.last_error())
    # accuracy: both calls' merged result against FP64 over the union of the candidate lists
    acc = accuracy(L, G, X, X2, torch.cat([a1, a2]), b, D, I, "fp64", nsample=512)
    kern = tr.get("fused_knn_simt")
    roof = None
    if kern and peaks.get("fp64_tflops"):
        kms = kern["ms"] / kern["launches"]
        ach = p.n * p.m * (2 * p.d + 3) / (kms * 1e-3) / 1e12
        roof = {"bound": "fp64", "achieved": ach, "peak": peaks["fp64_tflops"],
                "unit": "TFLOP/s", "frac": ach / peaks["fp64_tflops"], "kernel": "fused_knn_simt",
                "kernel_ms": kms, "peak_source": "measured FP64 DGEMM rate (peak_probes)"}
    # e2e: dgsknn through heap_t with host buffers, both calls per step
    h = G.Heap(p.n, p.k, 1.79e308, double=True)

    def host_step():
        h.D[:] = 1.79e308
        h.I[:] = -1
        G.gsknn_heap(p.k, p.X, p.X2, p.alpha, p.X, p.X2, p.beta, h)
        G.gsknn_heap(p.k, p.X, p.X2, alpha2, p.X, p.X2, p.beta, h)

    for _ in range(3):
        host_step()
    hs = max(10, args.steps)
    t0 = time.perf_counter()
    for _ in range(hs):
        host_step()
    th = (time.perf_counter() - t0) / hs
    h.free()
    # per call: the table's referenced row range with norms, both index lists, heaps both ways
    h2d = 2 * (N * (p.d + 1) * 8 + (p.n + p.m) * 4 + p.n * p.k * 12)
    d2h = 2 * p.n * p.k * 12
    res = {"workload": "plain dgsknn float64: N=8192 d=32 U[0,1), 4096 queries x 4096 "
                       "candidates, k=16, two merging calls per step",
           "value": evals / (ms * 1e-3), "unit": "distance-evals/s", "ms_per_step": ms,
           "kernels": tr, "roofline": roof, "accuracy": acc,
           "e2e": {"value": evals / th, "unit": "distance-evals/s", "ms_per_step": th * 1e3,
                   "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                   "api": "dgsknn (heap_t from heapCreate_d, host buffers)"}}
    if not args.no_cpu_baseline:
        try:
            res["cpu_baseline"] = config1_cpu_baseline(min(args.cpu_seconds, 10.0),
                                                      args.threads)
        except Exception as e:  # reported, not fatal
            res["cpu_baseline"] = {"error": str(e)[-400:]}
    return res

def run_ours(args, rank, world, local_rank):
    import torch
    from rnn_b200 import gsknn as G
    from rnn_b200 import workloads as W

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    L = G.lib()
    peaks = load_peaks()
    name2mode = {v: k for k, v in MODE_NAMES.items()}

    from rnn_b200 import replicas as RP
    barrier = RP.barrier

    out = {}
    if not args.profile_only and world == 1:
        probes = peak_probes(dev)
        peaks["tf32_tflops"] = probes["tf32_tflops"]
        peaks["fp64_tflops"] = probes["fp64_tflops"]
    if args.batch_only:
        return batching_form(L, G, W, dev, peaks, args, args.threads)
    if args.serve_only:
        return serving_form(L, G, W, dev, args)
    if not args.precision_only:
        p = W.config2(seed=2)
        nq = args.queries
        beta_h = RP.replica_queries(rank, world, N_POINTS, nq, default=p.beta)
        prob = DeviceProblem(p, beta_h, dev)
        clocks = ClockSampler(local_rank) if not args.profile_only else None
        mode = name2mode[args.mode]
        ms, trace = timed(L, G, prob, mode, args.steps, args.warmup, barrier, clocks)
        clk = clocks.stop() if clocks else None
        ms = RP.max_over_ranks(ms, device=dev)
        used = effective_mode_name(trace, p.d)
        value = RP.job_throughput(prob.evals, world, ms)
        out = {
            "metric": "distance-evals/s", "value": value, "unit": "distance-evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inputs; " + {"fp32": "fp32 CUDA-core distances",
                                       "tf32": "tf32 tensor distances + fp64 re-rank",
                                       "bf16": "bf16 tensor distances + fp64 re-rank",
                                       "bf16x3": "split-bf16 tensor distances + fp64 re-rank"}[used],
            "data": "synthetic (seeded gaussian mixture; no dataset published)",
            "mode": f"{args.mode} -> {used}",
            "exact_recall": used != "fp32",
            "config": {"workload": WORKLOAD, "points": N_POINTS, "d": D_DIM, "queries": nq,
                       "references": N_R, "k": K_NN, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (256 MiB point table gathered every step)"},
            "gpu_launches": sum(v["launches"] for v in trace.values()),
            "kernels": trace,
            "clocks": clk,
            "roofline": roofline(used, prob, trace, peaks, clk),
        }
        if args.profile_only:
            return out
        out["accuracy"] = accuracy(L, G, prob.X, prob.X2, prob.alpha, prob.beta, prob.D,
                                   prob.I, used)
        out["e2e"] = e2e_host(L, G, p, beta_h, args)
        if world == 1:
            modes = {}
            for nm in ("fp32", "tf32", "bf16", "bf16x3"):
                # plain BF16 at d = 64 overflows the band logs on this data; one step is enough
                steps = 2 if nm == "fp32" else 1 if nm == "bf16" else 5
                mms, tr = timed(L, G, prob, name2mode[nm], steps, 1)
                modes[nm] = {"ms_per_step": mms, "value": prob.evals / (mms * 1e-3),
                             "roofline": roofline(nm, prob, tr, peaks, clk),
                             "accuracy": accuracy(L, G, prob.X, prob.X2, prob.alpha,
                                                  prob.beta, prob.D, prob.I, nm)}
            out["modes"] = modes
        del prob
        torch.cuda.empty_cache()
    if world == 1:
        pf = precision_form(L, G, W, dev, peaks, args)
        if args.precision_only:
            return pf
        out["precision_form"] = pf
        if not args.profile_only:
            out["fp64_config1"] = fp64_config1(L, G, W, dev, peaks, args)
        if not args.no_batch and not args.profile_only:
            out["batching_form"] = batching_form(L, G, W, dev, peaks, args, args.threads)
        if not args.no_serve and not args.profile_only:
            out["serving_form"] = serving_form(L, G, W, dev, args)
    G.set_mode(0)
    return out


def effective_mode_name(trace, d):
    if "tc_knn" not in trace:
        return "fp32"
    from rnn_b200 import gsknn as G
    m = G.get_mode()
    if m == 0:
        return "bf16x3" if d <= 256 else "tf32"  # AUTO: split BF16 where its tiles fit
    return MODE_NAMES[m]


def precision_form(L, G, W, dev, peaks, args):
    """32,768 queries x 262,144 references, d = 256, k = 64, latent-manifold points."""
    import torch
    p = W.config3(seed=3)
    prob = DeviceProblem(p, np.ascontiguousarray(p.beta[:args.pf_queries]), dev)
    res = {"workload": f"precision form: queries={prob.nq} references=262144 d=256 k=64, "
                       "U[0,1)^8 latent through a seeded orthonormal basis + N(0,1e-3^2)"}
    name2mode = {v: k for k, v in MODE_NAMES.items()}
    wanted = args.pf_modes.split(",")
    for nm, steps in (("fp32", 2), ("tf32", 5), ("bf16", 5), ("bf16x3", 5)):
        if nm not in wanted:
            continue
        if args.precision_only and args.profile_only:
            steps = 1
        ms, tr = timed(L, G, prob, name2mode[nm], steps, 0 if args.profile_only else 1)
        res[nm] = {"ms_per_step": ms, "value": prob.evals / (ms * 1e-3),
                   "roofline": roofline(nm, prob, tr, peaks, None), "kernels": tr}
        if not args.profile_only:
            res[nm]["accuracy"] = accuracy(L, G, prob.X, prob.X2, prob.alpha, prob.beta,
                                           prob.D, prob.I, nm)
    if "fp32" in res:
        base = res["fp32"]["value"]
        for nm in ("tf32", "bf16", "bf16x3"):
            if nm in res:
                res[nm]["speedup_vs_plain_fp32"] = res[nm]["value"] / base
    if not args.precision_only and not args.no_cpu_baseline:
        try:
            res["cpu_baseline"] = slice_cpu_baseline("config3", args.threads)
        except Exception as e:  # reported, not fatal
            res["cpu_baseline"] = {"error": str(e)[-400:]}
    del prob
    torch.cuda.empty_cache()
    return res


def batching_form(L, G, W, dev, peaks, args, threads):
    """All-NN over randomized-tree leaves: 8 trees per pass x 4 passes, one persistent
    graph-replayed launch per pass."""
    import torch
    from rnn_b200 import batch as B
    p = W.config4(seed=4, n_points=args.batch_points, passes=args.batch_passes)
    T = p.trees_per_pass
    t0 = time.perf_counter()
    lv = B.rkdt_leaves(p.X, T * p.passes, p.leaf_min, p.leaf_max, seed=p.tree_seed)
    t_build = time.perf_counter() - t0
    passes = [lv.tree_range(i * T, (i + 1) * T) for i in range(p.passes)]
    evals = [float((np.diff(q.ptr).astype(np.float64) ** 2).sum()) for q in passes]
    Xd = torch.from_numpy(p.X).to(dev)
    X2d = torch.from_numpy(p.X2).to(dev)
    D = torch.full((p.N, p.k), float("inf"), device=dev)
    I = torch.full((p.N, p.k), -1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev)
    B.forget_tuning()
    job = B.BatchJob(Xd, X2d, D, I, p.k, T, p.leaf_min, shape=-1, stream=st)
    # warm-up: the first pass tunes the tile shape on its leaves and captures the graph
    job.run_pass(passes[0])
    job.sync()
    tune = job.info()
    D.fill_(float("inf"))
    I.fill_(-1)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(st)
    for q in passes:
        job.run_pass(q)
    ev1.record(st)
    job.sync()
    ms = ev0.elapsed_time(ev1)
    info = job.info()
    job.close()
    total = sum(evals)
    sm_mhz = 1965.0
    peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    achieved = total * (2 * p.d + 3) / (ms * 1e-3) / 1e12
    res = {
        "workload": p.name, "points": p.N, "d": p.d, "k": p.k, "trees_per_pass": T,
        "passes": p.passes, "leaves_per_pass": [int(q.nleaves) for q in passes],
        "evals_per_pass": evals, "tree_build_s": round(t_build, 2),
        "ms_total": ms, "ms_per_pass": ms / p.passes,
        "value": total / (ms * 1e-3), "unit": "distance-evals/s",
        "dtype": "f32 CUDA-core distances (sgsknn arithmetic)",
        "launch": {"tile_shape": info["shape_name"], "tile_rows": info["tile_rows"],
                   "persistent_grid": info["grid"], "work_items_last_pass": info["items"],
                   "autotune_ms": tune["tune_ms"], "cuda_graph": True,
                   "kernels_per_pass": 3},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": "nominal FP32 CUDA-core issue rate at 1965 MHz",
                     "note": "whole pass (pack + leaves + merge), 2d+3 flops per evaluation"},
    }
    del Xd, X2d, D, I
    torch.cuda.empty_cache()
    if args.stream_group > 0:
        res["streaming"] = streaming_form(B, p, passes, evals, args.stream_group)
    if not args.no_cpu_baseline:
        try:
            res["cpu_baseline"] = batch_cpu_baseline(max(5.0, args.cpu_seconds / 2), threads,
                                                     args.batch_points)
            res["speedup_vs_cpu"] = res["value"] / res["cpu_baseline"]["value"]
        except Exception as e:  # reported, not fatal
            res["cpu_baseline"] = {"error": str(e)[-400:]}
    return res


def streaming_form(B, p, passes, evals, group_points):
    """The same passes with the point table and the heaps in host memory (the streaming form,
    for point sets beyond HBM): groups of whole leaves of at most `group_points` points go
    through a device staging table. Host wall time per pass (the call blocks), after one warm-up
    pass."""
    D = np.full((p.N, p.k), np.inf, np.float32)
    I = np.full((p.N, p.k), -1, np.int32)
    job = B.StreamJob(p.X, p.X2.astype(np.float32), D, I, p.k, group_points=group_points,
                      leaf_min=p.leaf_min, shape=-1)
    job.run_pass(passes[0])  # warm-up: staging tuning, graph capture, first touch
    D.fill(np.inf)
    I.fill(-1)
    t0 = time.perf_counter()
    h2d = d2h = 0.0
    groups = 0
    for q in passes:
        job.run_pass(q)
        inf = job.info()
        h2d += inf["h2d_bytes"]
        d2h += inf["d2h_bytes"]
        groups += inf["groups"]
    sec = time.perf_counter() - t0
    job.close()
    return {"group_points": group_points, "groups_per_pass": groups / len(passes),
            "ms_per_pass": sec * 1e3 / len(passes), "value": sum(evals) / sec,
            "unit": "distance-evals/s",
            "h2d_bytes_per_pass": h2d / len(passes), "d2h_bytes_per_pass": d2h / len(passes),
            "note": "point table and heaps in host memory (numpy), host wall clock"}


def serving_form(L, G, W, dev, args):
    """Poisson request stream against a resident reference set (continuous batching)."""
    import threading
    import torch
    from rnn_b200 import serve as SV
    nref, d = args.serve_refs, 128
    R = W.uniform_table(5, nref, d).astype(np.float32)
    R2 = W.sq_norms(R)
    Rd = torch.from_numpy(R).to(dev)
    R2d = torch.from_numpy(R2).to(dev)
    del R
    rng = np.random.default_rng(55)
    n = args.serve_requests
    ms = np.floor(np.exp(rng.uniform(0.0, np.log(4096.0), size=n))).astype(int).clip(1, 4096)
    ks = rng.choice([8, 16, 64], size=n)
    qs = [W.uniform_table(5000 + i, int(ms[i]), d).astype(np.float32) for i in range(n)]
    serve_mode = {v: k for k, v in MODE_NAMES.items()}[args.serve_mode]
    srv = SV.Server(Rd, R2d, mode=serve_mode, max_batch_queries=8192, max_k=64,
                    heap_budget=2 << 30, slots=args.serve_slots, slice_rows=args.serve_slice)
    for m_w in (1, 128, 4096):  # warm-up: module loads, first launches of every kernel
        rid = srv.submit(W.uniform_table(99, m_w, d).astype(np.float32), 64)
        srv.wait(rid)
        srv.release(rid)
    def run_stream(count, rate, seed):
        """Poisson arrivals at `rate` per second; returns per-request stats and the wall time."""
        g = np.random.default_rng(seed)
        gaps = g.exponential(1.0 / rate, size=count)
        ids = [None] * count

        def arrivals():
            t = time.perf_counter()
            for i in range(count):
                t += gaps[i]
                dt = t - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                ids[i] = srv.submit(qs[i], int(ks[i]))

        lat, queue, rows, first = [], [], [], []
        t0 = time.perf_counter()
        th = threading.Thread(target=arrivals)
        th.start()
        for i in range(count):
            while ids[i] is None:
                time.sleep(0.0002)
            srv.wait(ids[i], timeout=120.0)
            st = srv.stats(ids[i])
            lat.append(st["total_ms"])
            queue.append(st["queue_ms"])
            rows.append(st["batch_rows"])
            first.append(st["batch"])
            srv.release(ids[i])
        t1 = time.perf_counter()
        th.join()
        return (np.asarray(lat), np.asarray(queue), np.asarray(rows), np.asarray(first),
                t1 - t0)

    def slowest(lat, queue, rows, first, mm, kk, count=5):
        """The slowest requests: arrival index, rows, k, latency, queue time, first batch."""
        order = np.argsort(-lat)[:count]
        return [{"i": int(i), "m": int(mm[i]), "k": int(kk[i]), "ms": round(float(lat[i]), 2),
                 "queue_ms": round(float(queue[i]), 2), "first_batch_rows": int(rows[i]),
                 "first_batch": int(first[i])} for i in order]

    def summary(lat, queue, mm):
        big = lat[mm >= 2048]
        return {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                "max": float(lat.max()),
                "p50_m_ge_2048": float(np.percentile(big, 50)) if big.size else None,
                "p99_m_ge_2048": float(np.percentile(big, 99)) if big.size else None,
                "queue_p50": float(np.percentile(queue, 50)),
                "queue_p99": float(np.percentile(queue, 99))}

    lat, queue, rows, first, wall = run_stream(n, args.serve_rate, 56)
    n_light = max(1, n // 2)
    lat_l, queue_l, rows_l, first_l, wall_l = run_stream(n_light, args.serve_rate / 3.0, 57)
    srv_mode, srv_probe = srv.mode, {k: round(v, 3) for k, v in srv.probe_ms.items()}
    srv.close()
    evals = float(ms.sum()) * nref
    res = {
        "workload": (f"serving: resident refs={nref} d={d} U[0,1); {n} requests, Poisson "
                     f"{args.serve_rate:g}/s, m log-uniform [1,4096] (mean {ms.mean():.0f}), "
                     f"k in {{8,16,64}}"),
        "dtype": (f"f32 inputs; {MODE_NAMES.get(srv_mode, srv_mode)} tensor distances + fp64 "
                  f"re-rank (exact top-k)" + (f" [auto: probe batch {srv_probe}]"
                                               if args.serve_mode == "auto" else "")),
        "latency_ms": summary(lat, queue, ms),
        "value": evals / wall, "unit": "distance-evals/s",
        "wall_s": wall, "mean_batch_rows": float(np.mean(rows)),
        "slice_rows": srv.slice_rows, "slots": args.serve_slots,
        "slowest": slowest(lat, queue, rows, first, ms, ks),
        "light_load": {"requests": n_light, "rate_per_s": args.serve_rate / 3.0,
                       "latency_ms": summary(lat_l, queue_l, ms[:n_light]),
                       "mean_batch_rows": float(np.mean(rows_l)),
                       "slowest": slowest(lat_l, queue_l, rows_l, first_l, ms[:n_light],
                                          ks[:n_light])},
        "p99_target_ms": 5.0,
    }
    # the same requests one at a time through the per-call entry point: plain FP32 CUDA-core
    # kernel and the per-call tensor-core path (which re-packs the reference set each call)
    sample = list(range(0, n, max(1, n // 24)))
    alpha = torch.arange(nref, dtype=torch.int32, device=dev)
    for name, mode in (("per_request_fp32", 1), ("per_request_tc", 0)):
        G.set_mode(mode)
        tot_e, tot_ms, lats = 0.0, 0.0, []
        for i in sample:
            Q = torch.from_numpy(qs[i]).to(dev)
            Q2 = torch.from_numpy(W.sq_norms(qs[i])).to(dev)
            beta = torch.arange(int(ms[i]), dtype=torch.int32, device=dev)
            k = int(ks[i])
            D = torch.full((int(ms[i]), k), float("inf"), device=dev)
            I = torch.full((int(ms[i]), k), -1, dtype=torch.int32, device=dev)
            st = torch.cuda.current_stream(dev)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
            rc = L.gsknn_s_device(nref, int(ms[i]), d, k, Rd.data_ptr(), R2d.data_ptr(), nref,
                                  alpha.data_ptr(), Q.data_ptr(), Q2.data_ptr(), int(ms[i]),
                                  beta.data_ptr(), D.data_ptr(), I.data_ptr(), k,
                                  st.cuda_stream)
            e1.record(st)
            torch.cuda.synchronize()
            if rc != 0:
                raise RuntimeError(G.last_error())
            t = e0.elapsed_time(e1)
            lats.append(t)
            tot_ms += t
            tot_e += float(ms[i]) * nref
        res[name] = {"requests": len(sample), "value": tot_e / (tot_ms * 1e-3),
                     "latency_ms_p50": float(np.percentile(lats, 50)),
                     "latency_ms_max": float(np.max(lats))}
    G.set_mode(0)
    res["speedup_vs_per_request_fp32"] = res["value"] / res["per_request_fp32"]["value"]
    del Rd, R2d
    torch.cuda.empty_cache()
    if not args.no_cpu_baseline:
        try:  # the reference's sgsknn on a request-sized query slice against the resident set
            cb = slice_cpu_baseline("config5", args.threads)
            cb["mean_request_ms"] = float(ms.mean()) * nref / cb["value"] * 1e3
            res["cpu_baseline"] = cb
        except Exception as e:  # reported, not fatal
            res["cpu_baseline"] = {"error": str(e)[-400:]}
    return res


def e2e_host(L, G, p, beta_h, args):
    import ctypes
    import torch
    nq = beta_h.size
    c_i = ctypes.c_int
    G.set_mode(0)
    steps = max(3, min(args.steps, 5))
    # one fresh pair of caller heaps (D = +inf, I = -1) per call, filled before the timed
    # region: the reset is the harness's, not part of the library call
    heaps = [(np.full((nq, K_NN), np.inf, dtype=np.float32),
              np.full((nq, K_NN), -1, dtype=np.int32)) for _ in range(steps + 1)]

    def call(D, I):
        L.sgsknn_var1(c_i(nq), c_i(N_R), c_i(D_DIM), c_i(K_NN), G._p(p.X), G._p(p.X2),
                      G._p(beta_h), G._p(p.X), G._p(p.X2), G._p(p.alpha), G._p(D), G._p(I))
        code, msg = G.last_error()
        if code != 0:
            raise RuntimeError(msg)

    call(*heaps[steps])  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(steps):
        call(*heaps[i])
    t = (time.perf_counter() - t0) / steps
    # bytes the library moves (gsknn_api.cu knn_host): the index lists, the heaps both ways, and
    # either the referenced rows alone (gathered on the host, when they cover under 60% of the
    # row range the lists reach) or that whole range of the table and its norms
    lo = int(min(beta_h.min(), p.alpha.min()))
    hi = int(max(beta_h.max(), p.alpha.max()))
    range_rows = hi - lo + 1
    n_idx = nq + N_R
    rows = n_idx if n_idx * 10 < range_rows * 6 else range_rows
    h2d = rows * (D_DIM + 1) * 4 + n_idx * 4 + 2 * nq * K_NN * 4
    d2h = 2 * nq * K_NN * 4
    return {"value": float(nq) * N_R / t, "unit": "distance-evals/s", "ms_per_step": t * 1e3,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "api": "sgsknn_var1 (host pointers, pageable numpy buffers), default mode"}




def kernel_case(name: str) -> dict:
    """One small invocation of one path (a warm-up call, then the call to profile), so that an
    ncu capture of any of the library's kernels can be taken on a small case; `last_ms` is the
    stream time of the profiled call (CUDA events around it):
      config1     dgsknn FP64 (pack_panels, fused_knn_simt<double>, finalize_heap)
      large_k     k = 600 float (dist_block, select_rows)
      tc_q8192    split BF16 on 8,192 headline queries (tc_pack, tc_knn, tc_rerank)
      fp32_q8192  plain FP32 on 8,192 headline queries (fused_knn_simt<float>)
      batch_small one pass of 8 trees over 262,144 mixture points (batch_pack, batch_knn_simt,
                  batch_merge); batch_small_tc the same in the tensor-core shape
      serve_one   one 512-row request against 1,048,576 resident points (query_norms,
                  scatter, the tensor-core kernels)"""
    import torch
    from rnn_b200 import gsknn as G
    from rnn_b200 import workloads as W
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    t = time.perf_counter()
    # device time of the last (profiled) call or pass
    ev = [torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]

    def dev_call(X, X2, alpha, beta, k, mode=0, reps=2):
        Xd, X2d = torch.from_numpy(X).to(dev), torch.from_numpy(X2).to(dev)
        a, b = torch.from_numpy(alpha).to(dev), torch.from_numpy(beta).to(dev)
        D = torch.empty((beta.size, k), dtype=Xd.dtype, device=dev)
        I = torch.empty((beta.size, k), dtype=torch.int32, device=dev)
        G.set_mode(mode)
        for _ in range(reps):
            D.fill_(float("inf"))
            I.fill_(-1)
            ev[0].record()
            G.knn_device(Xd, X2d, a, Xd, X2d, b, D, I)
            ev[1].record()
        torch.cuda.synchronize()
        G.set_mode(0)

    if name == "config1":
        p, _ = W.config1(1)
        dev_call(p.X, p.X2, p.alpha, p.beta, p.k)
    elif name == "large_k":
        p = W.config2(n_queries=2048, n_refs=65536, k=600)
        dev_call(p.X, p.X2, p.alpha, p.beta, p.k)
    elif name in ("tc_q8192", "fp32_q8192"):
        p = W.config2()
        beta = np.ascontiguousarray(p.beta[:8192])
        dev_call(p.X, p.X2, p.alpha, beta, p.k, mode=1 if name == "fp32_q8192" else 0)
    elif name in ("batch_small", "batch_small_tc"):
        from rnn_b200 import batch as B
        p = W.config4(n_points=1 << 18, passes=1)
        lv = B.rkdt_leaves(p.X, p.trees_per_pass, p.leaf_min, p.leaf_max, seed=p.tree_seed)
        Xd, X2d = torch.from_numpy(p.X).to(dev), torch.from_numpy(p.X2).to(dev)
        D = torch.full((p.N, p.k), float("inf"), device=dev)
        I = torch.full((p.N, p.k), -1, dtype=torch.int32, device=dev)
        job = B.BatchJob(Xd, X2d, D, I, p.k, p.trees_per_pass, p.leaf_min,
                         shape=3 if name == "batch_small_tc" else 2,
                         stream=torch.cuda.current_stream(dev))
        for _ in range(2):
            ev[0].record()
            job.run_pass(lv)
            ev[1].record()
        job.sync()
    elif name == "serve_one":
        from rnn_b200 import serve as SV
        R = W.uniform_table(61, 1 << 20, 128, np.float32)
        Rd = torch.from_numpy(R).to(dev)
        R2d = torch.from_numpy(W.sq_norms(R)).to(dev)
        srv = SV.Server(Rd, R2d, mode=0, max_batch_queries=1024, max_k=64, slots=1)
        Q = W.uniform_table(62, 512, 128, np.float32)
        for _ in range(2):
            ev[0].record()
            rid = srv.submit(Q, 64)
            srv.wait(rid)
            srv.release(rid)
            ev[1].record()
        srv.close()
    torch.cuda.synchronize()
    return {"kernel_case": name, "seconds": time.perf_counter() - t,
            "last_ms": ev[0].elapsed_time(ev[1])}

def summarize(out: dict) -> dict:
    """Compact figures of every leg, placed last in the JSON line so that a reader keeping only
    the tail of the line still has them."""
    def r(x, n=4):
        return None if x is None else float(f"{x:.{n}g}")
    sm = {}
    if "value" in out:
        sm["headline"] = {"evals_per_s": r(out["value"]), "ms": r(out.get("ms_per_step")),
                          "e2e_evals_per_s": r((out.get("e2e") or {}).get("value")),
                          "roofline_frac": r((out.get("roofline") or {}).get("frac")),
                          "mode": out.get("mode"),
                          "rows_exact": (out.get("accuracy") or {}).get("rows_exact_fp64_recall"),
                          "max_rel_dist_err": r((out.get("accuracy") or {}).get(
                              "max_rel_dist_err"), 3)}
    if "modes" in out:
        base = out["modes"]["fp32"]["value"]
        sm["modes"] = {nm: {"ms": r(v["ms_per_step"]),
                            "x_vs_fp32": r(v["value"] / base, 3),
                            "frac": r((v.get("roofline") or {}).get("frac"), 3),
                            "err_over_E": r((v.get("accuracy") or {}).get("max_err_over_E"), 3),
                            "rows_exact": (v.get("accuracy") or {}).get(
                                "rows_exact_fp64_recall")}
                       for nm, v in out["modes"].items()}
    pf = out.get("precision_form")
    if pf:
        sm["precision_form"] = {nm: {"ms": r(pf[nm]["ms_per_step"]),
                                     "x_vs_fp32": r(pf[nm].get("speedup_vs_plain_fp32"), 3),
                                     "frac": r((pf[nm].get("roofline") or {}).get("frac"), 3),
                                     "err_over_E": r((pf[nm].get("accuracy") or {}).get(
                                         "max_err_over_E"), 3),
                                     "max_rel_dist_err": r((pf[nm].get("accuracy") or {}).get(
                                         "max_rel_dist_err"), 3),
                                     "rows_exact": (pf[nm].get("accuracy") or {}).get(
                                         "rows_exact_fp64_recall")}
                                for nm in ("fp32", "tf32", "bf16", "bf16x3") if nm in pf}
        sm["precision_form"]["cpu_evals_per_s"] = r((pf.get("cpu_baseline") or {}).get("value"))
    c1 = out.get("fp64_config1")
    if c1:
        sm["fp64_config1"] = {"evals_per_s": r(c1["value"]), "ms": r(c1["ms_per_step"]),
                              "e2e_evals_per_s": r(c1["e2e"]["value"]),
                              "cpu_evals_per_s": r((c1.get("cpu_baseline") or {}).get("value")),
                              "frac": r((c1.get("roofline") or {}).get("frac"), 3),
                              "rows_exact": c1["accuracy"]["rows_exact_fp64_recall"]}
    bf = out.get("batching_form")
    if bf:
        sm["batching"] = {"evals_per_s": r(bf.get("value")), "ms_per_pass": r(
            bf.get("ms_per_pass")), "cpu_evals_per_s": r((bf.get("cpu_baseline") or {}).get(
                "value"))}
    sv = out.get("serving_form")
    if sv:
        lat = sv.get("latency_ms") or {}
        sm["serving"] = {"p50_ms": r(lat.get("p50")), "p99_ms": r(lat.get("p99")),
                         "evals_per_s": r(sv.get("value")),
                         "cpu_evals_per_s": r((sv.get("cpu_baseline") or {}).get("value")),
                         "cpu_mean_request_ms": r((sv.get("cpu_baseline") or {}).get(
                             "mean_request_ms"))}
    cb = out.get("cpu_baseline")
    if isinstance(cb, dict) and "value" in cb:
        sm["cpu_baseline_evals_per_s"] = r(cb["value"])
    return sm

def main():
    args = parse()
    if args.cpu_worker:
        cpu_worker(args.cpu_worker)
        return
    if args.kernel_case:
        print(json.dumps(kernel_case(args.kernel_case)), flush=True)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()

    if args.impl == "reference":
        # the reference's CPU implementation of the path; rank 0 alone
        if rank != 0:
            return
        # each step is a bounded sample (a query slice against all references), sized so the
        # whole --steps K --warmup W run takes about a minute
        steps, warmup = max(1, args.steps), max(0, args.warmup)
        per_step = max(0.5, min(args.cpu_seconds, 60.0 / (steps + warmup)))
        cb = cpu_baseline(per_step, threads, steps=steps, warmup=warmup)
        out = {"impl": "reference", "metric": "distance-evals/s", "value": cb["value"],
               "unit": "distance-evals/s", "n_gpus": args.gpus, "steps": steps,
               "warmup": warmup, "ms_per_step": cb["ms_per_step"],
               "higher_is_better": True, "scaling": "weak",
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
    args.threads = threads
    out = run_ours(args, rank, world, local_rank)
    if (rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile_only
            and not args.precision_only and not args.batch_only and not args.serve_only):
        try:
            out["cpu_baseline"] = cpu_baseline(args.cpu_seconds, threads)
        except Exception as e:  # reported, not fatal
            out["cpu_baseline"] = {"error": str(e)[-400:]}
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        if world == 1 and not args.profile_only:
            out["summary"] = summarize(out)
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
