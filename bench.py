"""Benchmark: batched complex64 2D BWPM solves per second on one B200 (or N replicas).

Workload (seeded, synthetic): 256 tilted-slab 2D solves of uneven size (ny 256-8192 including
3·2^k, nz 100-2000 slabs, λ 0.4-1.0 µm, 0-30° incidence, n 1.4-1.8, 0-8° tilted front face,
absorbing mask, TE/TM alternating, 6 bidirectional iterations); bwpm_b200.workloads.batch2d.
A step is one solve of the whole batch. `value` is solves/s with inputs resident on the device;
`e2e` is the same through the public batch API with host copies of the incident fields and of
the transmitted/reflected results inside the timed region.

Beside it: p50/p99 per-solve device latency, the plain per-solve FP64 GPU path (the drop-in
CudaSolver) on a seeded sample of the same batch with the relative L2 error of the batched
complex64 results against it, the roofline of the resident kernel, and the reference CPU core
(oracle/_ref, built from the reference's own sources) on a bounded sample, all host cores.

--impl reference: times the reference CPU implementation on the same workload and metric.
Multi-GPU (torchrun): replicas only, every rank solves its own copy of the batch.
"""

from __future__ import annotations

import argparse
import gc
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "solves/s (batched complex64 2D BWPM, 256 uneven solves, 6 iterations)"
WORKLOAD = ("batched-2d: 256 seeded tilted-slab solves, ny 256-8192 incl. 3*2^k, nz 100-2000, "
            "lambda 0.4-1.0 um, 0-30 deg incidence, n 1.4-1.8, 0-8 deg tilt, mask, TE/TM, "
            "6 iterations")
COUNT, SEED = 256, 4
REDUCED: dict = {}  # set by --reduced (profiling runs); empty for the benchmark itself
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # SMs × FP32 lanes × FMA × max clock
# DRAM bytes (read + write) of the class kernels of one batched run of this workload, summed
# over the classes (dram__bytes_read.sum + dram__bytes_write.sum of an earlier full-workload
# capture of these kernels; the reduced-case capture gives a few KB per slab step); the fields
# stay on chip, this is mostly pair-id planes of the longest lines that L2 cannot hold
TRAFFIC_PER_RUN_BYTES = 1.82e9


def _dist():
    from bwpm_b200 import replicas

    dist, rank, ws, _ = replicas.init("nccl")
    return dist, rank, ws


def _max_over_ranks(dist, x: float) -> float:
    from bwpm_b200 import replicas

    return replicas.max_over_ranks(dist, x)


def _barrier(dist):
    from bwpm_b200 import replicas

    replicas.barrier(dist)


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int, period_ms: int = 100):
        self.device = device
        self.period_ms = period_ms
        self.rows: list[list[str]] = []
        self._p = None
        self._t = None

    def _read(self):
        for line in self._p.stdout:
            line = line.strip()
            if line:
                self.rows.append([c.strip() for c in line.split(",")])

    def __enter__(self):
        # one nvidia-smi streaming a sample every period_ms (a process per sample would take
        # longer than the sampling period itself)
        try:
            self._p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            t0 = time.perf_counter()  # the sampler is live before the timed region starts
            while not self.rows and self._p.poll() is None and time.perf_counter() - t0 < 2.0:
                time.sleep(0.01)
        except Exception:  # noqa: BLE001 - sampling is best effort (no nvidia-smi: no samples)
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is not None:
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._p.kill()
        if self._t is not None:
            self._t.join(timeout=5)

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---- CPU reference (oracle/_ref: the reference's own C++ CPU core) ---------------------------

_CPU_CORE = None


def _ref_kind() -> str:
    return "reference" if sorted((ROOT / "oracle" / "_ref").glob("_core*.so")) else "port"


def _cpu_solve(args):
    """One solve on the reference CPU core (1 thread) or, without it, the numpy oracle port;
    returns the solve's own time in s."""
    global _CPU_CORE
    prm, kind = args
    from bwpm_b200 import workloads

    p = workloads.tilted_slab2d_from(prm)
    if kind == "reference" and _CPU_CORE is None:
        import importlib.util

        so = sorted((ROOT / "oracle" / "_ref").glob("_core*.so"))[0]
        spec = importlib.util.spec_from_file_location("_core", so)
        _CPU_CORE = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_CPU_CORE)
    t0 = time.perf_counter()
    if kind == "reference":
        _CPU_CORE.Solver(*p.core_args(), 1).run(p.field, p.iterations, [])
    else:
        from oracle import port

        port.Solver(*p.core_args()).run(p.field, p.iterations)
    return time.perf_counter() - t0


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _cost(prm: dict) -> float:
    """Estimated single-thread cost of one solve: ∝ N·log2 N per slab-pass."""
    return prm["ny"] * np.log2(prm["ny"]) * prm["nz"] * 2 * max(prm["iterations"], 1)


class CpuReference:
    """The reference CPU implementation on the host cores: one single-threaded solve per core
    (a process pool, spawned before any GPU work of this process), timed by the wall clock.

    Slice k is `per_step` instances of a seeded permutation of the batch (the slices rotate over
    the whole batch); `steps(k0, count)` solves `count` consecutive slices and returns (solves,
    wall seconds)."""

    def __init__(self, params: list[dict], per_step: int | None = None):
        import multiprocessing as mp

        self.params = params
        self.kind = _ref_kind()
        self.cores = os.cpu_count() or 1
        self.per_step = per_step or 3 * self.cores
        self.order = [int(i) for i in np.random.default_rng(123).permutation(len(params))]
        self.pool = mp.get_context("spawn").Pool(self.cores)

    def warm(self) -> None:
        """Loads the core in every worker (one small solve each)."""
        small = min(self.params, key=_cost)
        self.pool.map(_cpu_solve, [(small, self.kind)] * self.cores, chunksize=1)

    def slice(self, k: int) -> list[int]:
        n = len(self.order)
        idx = [self.order[(k * self.per_step + j) % n] for j in range(self.per_step)]
        return sorted(idx, key=lambda i: -_cost(self.params[i]))

    def steps(self, k0: int, count: int) -> tuple[int, float]:
        """Solves the slices of steps k0 … k0 + count − 1 as one stream of work on the pool (the
        cores stay busy across step boundaries, as a throughput run would keep them; longest
        first); returns (solves, wall seconds)."""
        idx = [i for k in range(k0, k0 + count) for i in self.slice(k)]
        jobs = [(self.params[i], self.kind) for i in sorted(idx, key=lambda i: -_cost(self.params[i]))]
        t0 = time.perf_counter()
        for _ in self.pool.imap_unordered(_cpu_solve, jobs, chunksize=1):
            pass
        return len(jobs), time.perf_counter() - t0

    def close(self) -> None:
        self.pool.close()
        self.pool.join()

    def describe(self, steps: int) -> str:
        return (f"{steps} steps of {self.per_step} seeded instances each (slices of a seeded "
                f"permutation of the {len(self.params)}-solve batch), solved as one stream "
                f"(longest first), one single-threaded solve per core in {self.cores} processes "
                f"on {cpu_model()}; value = solves / wall time, both measured")


def cpu_baseline(ref: CpuReference, steps: int = 2) -> dict:
    """Reference CPU throughput on a bounded sample of the batch, all host cores."""
    ref.warm()
    done, wall = ref.steps(0, steps)
    return {"value": done / wall, "unit": "solves/s", "cores": ref.cores, "kind": ref.kind,
            "cpu": cpu_model(), "sample": ref.describe(steps)}


def _config(ws: int, count: int = COUNT) -> dict:
    """The workload's config, identical in both arms."""
    return {"workload": WORKLOAD if not REDUCED else f"REDUCED profiling case {REDUCED}",
            "global_batch": count * ws, "seq_len": None, "parallelism": f"replicas{ws}",
            "l2": "GPU arm: flushed (512 MB write) before each timed step; CPU arm: n/a"}


def run_reference(args) -> None:
    """The reference arm: the reference's own CPU core (oracle/_ref, built from its sources) on
    the host cores, each step a measured slice of the workload. Rank 0 alone runs it."""
    dist, rank, ws = _dist_for_reference()
    if rank != 0:
        return
    params = _params()
    ref = CpuReference(params, per_step=args.ref_sample or None)
    ref.warm()
    for _ in range(args.warmup - 1):  # the first warm-up step loaded the core in every worker
        ref.warm()
    done, wall = ref.steps(0, args.steps)
    ref.close()
    v = done / wall
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded)", "config": _config(ws, len(params)), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": ref.cores, "kind": ref.kind,
                             "cpu": cpu_model(), "sample": ref.describe(args.steps)},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": f"a step solves {ref.per_step} of the {COUNT} solves; the timed steps run as "
                    "one stream on the pool; ms_per_step = measured wall time / steps; value = "
                    "all solves of the timed steps / that wall time"}
    print(json.dumps(line), flush=True)


def _dist_for_reference():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return None, rank, ws


def _params():
    from bwpm_b200 import workloads

    prm = workloads.batch2d_params(COUNT, SEED)
    if REDUCED:  # reduced case for profiling: fewer solves, shorter chains, optionally one length
        prm = [dict(p, nz=min(p["nz"], REDUCED["nz_max"]), iterations=REDUCED["iterations"],
                    ny=REDUCED.get("ny") or p["ny"])
               for p in prm[: REDUCED["count"]]]
    return prm


# ---- our arm ----------------------------------------------------------------------------------

def run_ours(args) -> None:
    dist, rank, ws = _dist()
    device = int(os.environ.get("LOCAL_RANK", "0")) if dist else 0
    from bwpm_b200 import _core, replicas, workloads
    from bwpm_b200.batch import Batch2D, flush_l2, host_register, host_unregister
    from bwpm_b200.model import Grid2D, power_flux

    params = _params()
    t_setup = time.perf_counter()
    b = Batch2D(device)
    if args.variants:  # profiling: the kernel choice of an earlier (timed) run, no autotuning
        for spec in args.variants.split(","):
            ny, v = spec.split(":")
            b.set_variant(int(ny), int(v))
    else:
        b.set_autotune(True)  # kernel variant per length chosen by measurement at prepare
    fields = []
    for prm in params:
        p = workloads.tilted_slab2d_from(prm)
        b.add_problem(p)
        fields.append(p.field[:, 0, :].copy())
        del p
    b.prepare()
    setup_s = time.perf_counter() - t_setup
    stats = b.stats()
    work = b.work()
    packed_in = np.ascontiguousarray(np.concatenate([f.ravel() for f in fields]))
    packed_out = np.empty(2 * packed_in.size, dtype=np.complex128)
    host_register(packed_in)
    host_register(packed_out)
    for _ in range(args.warmup):
        b.run()
    _barrier(dist)
    times = []
    with Clocks(device) as clk:
        for _ in range(args.steps):
            flush_l2(device)
            _barrier(dist)
            times.append(b.run())
    clocks = clk.summary()
    step_ms = _max_over_ranks(dist, float(np.sum(times))) / args.steps
    count = len(params)
    lat = np.array([b.result(i)["latency_ms"] for i in range(count)])
    # end to end through the public API: H2D of incident fields, solve, D2H of results
    e2e_times = []
    for _ in range(max(1, args.warmup // 2)):
        b.solve_packed(packed_in, packed_out)
    for _ in range(args.steps):
        flush_l2(device)
        e2e_times.append(b.solve_packed(packed_in, packed_out))
    e2e_ms = _max_over_ranks(dist, float(np.mean(e2e_times)))
    host_unregister(packed_in)
    host_unregister(packed_out)
    if rank != 0:
        _barrier(dist)
        return
    value = replicas.throughput(ws, count, step_ms)
    # plain per-solve FP64 GPU path (drop-in CudaSolver) on a seeded sample; L2 error of the
    # batched complex64 results against it
    rng = np.random.default_rng(7)
    sample = [int(i) for i in rng.permutation(count)[: args.fp64_sample]]
    fp64_t, errs, eps_err, eps_div = [], [], [], []
    ref_cuda = _reference_cuda_core()
    ref_t, ref_diff = [], []
    for i in sample:
        p = workloads.tilted_slab2d_from(params[i])
        s = _core.CudaSolver(*p.core_args(), device)
        t0 = time.perf_counter()
        r64 = s.run(p.field, p.iterations, [])
        fp64_t.append(time.perf_counter() - t0)
        if ref_cuda is not None:  # the reference's own GPU core (cuFFT, FP64) on the same solve
            rs = ref_cuda.CudaSolver(*p.core_args(), device)
            t0 = time.perf_counter()
            rr = rs.run(p.field, p.iterations, [])
            ref_t.append(time.perf_counter() - t0)
            ref_diff.append(max(_rel(r64[k], rr[k]) for k in ("transmitted", "reflected")))
            del rs, rr
        r32 = b.result(i)
        for key in ("transmitted", "reflected"):
            ref = r64[key][:, 0]
            errs.append(float(np.linalg.norm(r32[key] - ref) / max(np.linalg.norm(ref), 1e-300)))
        g = Grid2D(p.ny, p.dy, p.dz, prm_wl(params[i]))
        p_in = power_flux(p.field[:, 0], g, p.index_before)
        last = complex(p.indices[int(p.labels[-1, p.ny // 2, 0])])
        inst_err, eps64 = [], []
        for k in range(p.iterations):
            pt = power_flux(r64["transmitted_iter"][k][:, 0], g, last)
            pr = power_flux(r64["reflected_iter"][k][:, 0], g, p.index_before, direction=-1)
            eps64.append(1.0 - (pt + pr) / p_in)
            # energy balance error relative to the largest flux involved
            inst_err.append(abs(r32["energy_residual"][k] - eps64[-1]) / max(1.0, (pt + pr) / p_in))
        # an instance whose FP64 iteration diverges (|ε| above 1: light trapped in the tilted
        # slab grows from iteration to iteration) has no energy balance to match
        (eps_div if max(abs(e) for e in eps64) > 1.0 else eps_err).append(max(inst_err))
        del s
    mean_cost = np.mean([prm["ny"] * np.log2(prm["ny"]) * prm["nz"] for prm in params])
    samp_cost = np.mean([params[i]["ny"] * np.log2(params[i]["ny"]) * params[i]["nz"] for i in sample]) if sample else 1.0
    fp64_rate = 1.0 / (np.mean(fp64_t) * mean_cost / samp_cost) if sample else None
    ref_cuda_rate = 1.0 / (np.mean(ref_t) * mean_cost / samp_cost) if ref_t else None
    # roofline of the resident kernel: algorithmic FLOPs per launch ÷ launch time
    kern_s = step_ms * 1e-3
    achieved = work["flops"] / kern_s / 1e12
    hbm_peak = _peak("hbm_gbs")
    kernels = [f"{c['ny']}:{c['threads']}t x{c['cluster']} v{c['variant']}" for c in b.classes()]
    del b  # the batched engine's device pools and streams are released before the other sections
    gc.collect()
    served = run_served(device, args.served_fp64) if not args.no_served else None
    configs = None
    if not args.no_configs:
        try:
            configs = run_configs(device)
        except Exception as e:  # noqa: BLE001 - a side measurement must not cost the headline
            configs = {"error": f"{type(e).__name__}: {e}"}
    cb = None
    if not args.no_cpu:
        ref = CpuReference(params)
        cb = cpu_baseline(ref, steps=2)
        ref.close()
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic (seeded)",
        "config": _config(ws, count),
        "engine": {"work_items": stats["work_items"], "classes": stats["classes"],
                   "kernels": kernels},
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "fp64_plain": {"value": fp64_rate, "unit": "solves/s", "sample": len(sample),
                       "note": "per-solve FP64 CudaSolver (drop-in path), mean sample time scaled "
                               "to the batch's mean N·log2N·nz",
                       "speedup_batched_c64": value / ws / fp64_rate if fp64_rate else None,
                       "reference_cuda_core": {
                           "value": ref_cuda_rate, "unit": "solves/s",
                           "note": "the reference's own CudaSolver (cuFFT, FP64; built for "
                                   "sm_100a from its sources) on the same sample and scaling",
                           "rel_l2_vs_ours_fp64_max": max(ref_diff) if ref_diff else None,
                           "speedup_batched_c64": value / ws / ref_cuda_rate
                           if ref_cuda_rate else None}},
        "l2_err_max": float(np.max(errs)) if errs else None,
        "eps_err_max": float(np.max(eps_err)) if eps_err else None,
        "eps_err_note": "|eps_c64 - eps_fp64| / max(1, (P_R + P_T)/P_in) over the iterations of the "
                        "sample's instances whose FP64 iteration converges; "
                        f"{len(eps_div)} sampled instance(s) diverge in FP64 (|eps| > 1)",
        "eps_err_max_divergent": float(np.max(eps_div)) if eps_div else None,
        "e2e": {"value": ws * count / (e2e_ms * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": int(packed_in.nbytes), "d2h_bytes_per_step": int(packed_out.nbytes)},
        "gpu_launches": int(stats["classes"]) * args.steps,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": FP32_NOMINAL_TFLOPS,
                     "unit": "TFLOP/s", "frac": achieved / FP32_NOMINAL_TFLOPS,
                     "traffic": TRAFFIC_PER_RUN_BYTES if not REDUCED else None,
                     "traffic_note": "bytes per batched run (all class kernels), from an earlier "
                                     "full-workload ncu capture of these kernels; a reduced-case "
                                     "capture gives ~13 KB per 8192-point slab step",
                     "note": "shared-memory FFT: SIMT FP32 and shared-memory bound, no tensor "
                             "cores (FFT is not a dense contraction); peak = nominal FP32 "
                             "(no measured FP32 peak in MEASURED_PEAKS.json)",
                     "hbm": {"achieved": work["bytes"] / kern_s / 1e9, "peak": hbm_peak,
                             "unit": "GB/s", "frac": work["bytes"] / kern_s / 1e9 / hbm_peak,
                             "peak_source": _peak_source()}},
        "served": served,
        "configs": configs,
        "cpu_baseline": cb,
        "clocks": clocks,
        "setup_s": setup_s,
        "device_bytes": stats["device_bytes"],
    }
    # the figures a reader of the line's tail needs, last
    line["summary"] = _summary(line)
    print(json.dumps(line), flush=True)
    _barrier(dist)


def _summary(line: dict) -> dict:
    """A compact digest of the line (parity, the FP64 and CPU comparisons, served, configs)."""
    def get(d, *keys):
        for k in keys:
            if not isinstance(d, dict):
                return None
            d = d.get(k)
        return d

    cfg = line.get("configs") or {}
    return {
        "solves_per_s": line["value"], "e2e_solves_per_s": get(line, "e2e", "value"),
        "l2_err_max_vs_fp64": line.get("l2_err_max"), "eps_err_max_vs_fp64": line.get("eps_err_max"),
        "speedup_vs_fp64_plain": get(line, "fp64_plain", "speedup_batched_c64"),
        "speedup_vs_reference_cuda_fp64": get(line, "fp64_plain", "reference_cuda_core",
                                              "speedup_batched_c64"),
        "cpu_reference_solves_per_s": get(line, "cpu_baseline", "value"),
        "fp32_frac": get(line, "roofline", "frac"),
        "served_solves_per_s": get(line, "served", "solves_per_s"),
        "served_p50_p99_ms": [get(line, "served", "p50_ms"), get(line, "served", "p99_ms")],
        "served_speedup_vs_fp64": get(line, "served", "speedup_vs_fp64_plain"),
        "slab2d_ms_c64_both_fp64_each": [get(cfg, "slab2d", "c64_batched_ms_both"),
                                       get(cfg, "slab2d", "fp64_ms_per_solve")],
        "born2d_s_c64_fp64": [get(cfg, "born2d", "c64_s"), get(cfg, "born2d", "fp64_s")],
        "microlens3d_s_c64_fp64_refcuda": [get(cfg, "microlens3d", "c64_s"), get(cfg, "microlens3d", "fp64_s"),
                                    get(cfg, "microlens3d", "reference_cuda_fp64_s")],
    }


# ---- served request stream (continuous batching) ----------------------------------------------

SERVED_COUNT, SERVED_MAX3D = 48, 1024


def _rel_floor(a, b, floor: float) -> float:
    """‖a − b‖ / max(‖b‖, floor): relative error that stays meaningful for a vanishing field."""
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(b)), floor, 1e-300))


def _rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_served(device: int, fp64_sample: int) -> dict:
    """The served configuration: seeded Poisson arrivals of 70 % 2D (ny 1024-4096, 500-2000 slabs)
    and 30 % 3D (lateral up to SERVED_MAX3D², 200-600 slabs) solves, microlens arrays or tilted
    fibre facets, 2 iterations. Closed-loop passes (all requests at t = 0; the median of three)
    measure capacity; the open-loop pass offers 80 % of it as Poisson arrivals and reports
    p50/p99 latency (submit -> result on the host) and solves/s; the plain FP64 per-solve path is
    timed on a sample."""
    from bwpm_b200 import _core, workloads
    from bwpm_b200.serve import Server, serve_stream

    # 3D requests carry their geometry, not a label volume: their labels are generated on the
    # device (a 1024² × 600 volume would be 2.5 GB of int32 labels on the host)
    stream = workloads.request_stream(SERVED_COUNT, 1.0, seed=5, iterations=2,
                                      max_lateral_3d=SERVED_MAX3D, host_labels=False)
    probs = [p for _, p in stream]
    with Server(device) as srv:  # warm-up: module loading and first-use set-up of both engines
        serve_stream(srv, [(0.0, p) for p in (next(p for p in probs if p.nx == 1),
                                              next(p for p in probs if p.nx != 1))])
    walls = []
    for _ in range(3):  # closed loop: capacity, the median of three passes (host-bound, noisy)
        with Server(device) as srv:
            _, wall = serve_stream(srv, [(0.0, p) for p in probs])
        walls.append(wall)
    capacity = len(probs) / float(np.median(walls))
    rate = 0.8 * capacity
    arrivals = workloads.poisson_arrivals(len(probs), rate, seed=5)
    with Server(device) as srv:
        res, wall = serve_stream(srv, list(zip(arrivals, probs)))
        st = srv.stats()
    lat = np.array([r["latency_ms"] for r in res])
    # plain FP64 per-solve path (drop-in CudaSolver) on a sample; L2 error of the served results
    rng = np.random.default_rng(9)
    sample = [int(i) for i in rng.permutation(len(probs))[:fp64_sample]]
    t64, errs, errs_div, detail = [], [], [], []
    for i in sample:  # a per-solve user pays the solver's set-up and its run
        p = probs[i]
        t0 = time.perf_counter()
        if p.nx == 1:
            s = _core.CudaSolver(*p.core_args(), device)
        else:  # FP64 with the labels generated on the device too (no host volume)
            s = _core.CudaSolver.from_geometry(p.ny, p.nx, p.dy, p.dx, p.dz, p.k0, p.indices,
                                               p.geometry, p.index_before, p.mask, device)
        r64 = s.run(p.field, p.iterations, [])
        t64.append(time.perf_counter() - t0)
        del s
        err = max(_rel(res[i][key], r64[key][:, 0] if p.nx == 1 else r64[key])
                  for key in ("transmitted", "reflected"))
        # growth of the reflected field from one iteration to the next in FP64: a request whose
        # iteration diverges (light trapped by a tilted facet grows each iteration, in the
        # reference's algorithm as here) has no converged field for complex64 to match
        norms = [float(np.linalg.norm(x)) for x in r64["reflected_iter"]]
        growth = max((b / a for a, b in zip(norms, norms[1:]) if a > 0), default=1.0)
        diverges = growth > 1.1 or norms[-1] > float(np.linalg.norm(p.field))
        (errs_div if diverges else errs).append(err)
        detail.append({"request": i, "name": p.name, "ny": p.ny, "nx": p.nx, "nz": p.nz,
                       "l2_err": err, "reflected_growth": growth, "diverges": diverges})
    fp64_rate = 1.0 / float(np.mean(t64)) if t64 else None
    value = len(probs) / wall
    return {
        "requests": len(probs), "n_3d": sum(p.nx != 1 for p in probs),
        "solves_per_s": value, "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "offered_rate_hz": rate, "closed_loop_solves_per_s": capacity,
        "fp64_plain_solves_per_s": fp64_rate, "fp64_sample": len(sample),
        "speedup_vs_fp64_plain": value / fp64_rate if fp64_rate else None,
        "capacity_speedup_vs_fp64_plain": capacity / fp64_rate if fp64_rate else None,
        "l2_err_max": float(np.max(errs)) if errs else None,
        "l2_err_note": "max over the FP64 sample's requests whose iteration converges (reflected "
                       "field growing by at most 10 % per iteration and below the incident one)",
        "l2_err_max_divergent": float(np.max(errs_div)) if errs_div else None,
        "n_divergent_in_sample": len(errs_div),
        "sample_detail": detail,
        "launch_groups": st["groups"], "max_concurrent": st["max_concurrent"],
        "peak_device_bytes": st["peak_bytes"],
        "note": "seeded Poisson stream at 80 % of the measured closed-loop capacity; 3D lateral "
                f"sizes 256^2-{SERVED_MAX3D}^2 with labels generated on the device; latency = "
                "submit -> result on the host; fp64 = per-solve FP64 CudaSolver (set-up + run; "
                "3D from the same geometry) on the sample, "
                "sequential; solves_per_s is bounded by the offered load, the closed-loop passes "
                "(all requests at once; median of three) give the capacity",
    }


# ---- the other configurations (parity and timing beside the headline; not part of its value) ----

_REF_CORE: dict = {}


def _reference_core():
    """The reference's compiled bwpm._core, loaded once per process: the staged install in
    baseline/_ref (oracle/stage_reference.sh; CPU Solver and its own CUDA core) where present,
    else the CPU core of oracle/_ref; None when neither exists. (Both register the same C++
    types with pybind11, so only one of them can be loaded in a process.)"""
    if "core" not in _REF_CORE:
        import importlib.util

        mod = None
        for d in (ROOT / "baseline" / "_ref" / "bwpm", ROOT / "oracle" / "_ref"):
            so = sorted(d.glob("_core*.so"))
            if not so:
                continue
            try:
                spec = importlib.util.spec_from_file_location("_core", so[0])
                mod = importlib.util.module_from_spec(spec)
                spec.loader.exec_module(mod)
                break
            except ImportError:
                mod = None
        _REF_CORE["core"] = mod
    return _REF_CORE["core"]


def _reference_cuda_core():
    """The reference core when it has its CUDA backend (the staged install), else None."""
    mod = _reference_core()
    return mod if mod is not None and getattr(mod, "HAS_CUDA", False) else None


def run_configs(device: int) -> dict:
    """The slab, Born and microlens workloads on this GPU: the complex64 result of this
    implementation against the per-solve FP64 drop-in path (time and relative L2 error), the
    reference's own GPU core (cuFFT, FP64; staged build) on the same solves, and for the 2D slab
    the reference's CPU core on one thread. The Born chain runs at full size in TE; times include set-up."""
    from bwpm_b200 import _core, workloads
    from bwpm_b200.batch import Batch2D

    def timed(fn):
        t0 = time.perf_counter()
        r = fn()
        return r, time.perf_counter() - t0

    ref_core = _reference_core()
    ref_cuda = _reference_cuda_core()
    out: dict = {}
    # 1: 5 um slab, 1024 points, 250 slabs, 8 iterations, TE and TM
    probs = [workloads.slab2d("te"), workloads.slab2d("tm")]
    b = Batch2D(device)
    ids = [b.add_problem(p) for p in probs]
    b.prepare()
    b.run()
    batch_ms = b.run()
    t64, tcpu, tref, errs = [], [], [], []
    for p, i in zip(probs, ids):
        r64, dt = timed(lambda p=p: _core.CudaSolver(*p.core_args(), device).run(p.field, p.iterations, []))
        t64.append(dt)
        r32 = b.result(i)
        errs += [_rel(r32["transmitted"], r64["transmitted"][:, 0]),
                 _rel(r32["reflected"], r64["reflected"][:, 0])]
        if ref_core is not None:
            _, dt = timed(lambda p=p: ref_core.Solver(*p.core_args(), 1).run(p.field, p.iterations, []))
            tcpu.append(dt)
        if ref_cuda is not None:
            _, dt = timed(lambda p=p: ref_cuda.CudaSolver(*p.core_args(), device).run(p.field, p.iterations, []))
            tref.append(dt)
    out["slab2d"] = {"solves": 2, "c64_batched_ms_both": batch_ms,
                     "fp64_ms_per_solve": 1e3 * float(np.mean(t64)),
                     "reference_cuda_fp64_ms_per_solve": 1e3 * float(np.mean(tref)) if tref else None,
                     "cpu_reference_ms_per_solve": 1e3 * float(np.mean(tcpu)) if tcpu else None,
                     "cpu_threads": 1, "l2_err_max": float(np.max(errs)),
                     "workload": "1024 points, 250 slabs of lambda/10, 5 um slab n=1.5 in air, "
                                 "8 iterations, TE and TM"}
    del b
    # 3: microlens with a tilted silver back face, 512^2 points, 400 slabs, 6 iterations
    p = workloads.microlens3d()
    points_passes = p.ny * p.nx * p.nz * 2 * p.iterations
    s32, t32_setup = timed(lambda: _core.CudaSolver(*p.core_args(), device, precision=32))
    r32, t32 = timed(lambda: s32.run(p.field, p.iterations, []))
    del s32
    s64, t64_setup = timed(lambda: _core.CudaSolver(*p.core_args(), device))
    r64, t64s = timed(lambda: s64.run(p.field, p.iterations, []))
    del s64
    tref3 = None
    if ref_cuda is not None:
        _, tref3 = timed(lambda: ref_cuda.CudaSolver(*p.core_args(), device).run(p.field, p.iterations, []))
    # the silver fills everything behind the back face: the transmitted field is ~1e-94 of the
    # incident one in FP64, below the complex64 range, so errors are relative to the larger of
    # the field's own norm and 1e-6 of the incident field's
    floor = 1e-6 * float(np.linalg.norm(p.field))
    out["microlens3d"] = {"c64_s": t32_setup + t32, "c64_run_s": t32, "fp64_s": t64_setup + t64s,
                          "fp64_run_s": t64s,
                          "reference_cuda_fp64_s": tref3,
                          "l2_err": max(_rel_floor(r32["transmitted"], r64["transmitted"], floor),
                                        _rel_floor(r32["reflected"], r64["reflected"], floor)),
                          "l2_err_reflected": _rel(r32["reflected"], r64["reflected"]),
                          "transmitted_norm_over_incident": float(np.linalg.norm(r64["transmitted"])) /
                                                            float(np.linalg.norm(p.field)),
                          "workload": "512^2 points, 400 slabs of lambda/8, lens n=1.52 + silver, "
                                      "6 iterations; *_s include set-up (labels -> step tables)"}
    # seconds per grid point and pass (one direction of one iteration): the runtime model of
    # the reference's adapter (src/bwpm/adapter.py:35), measured on this configuration
    out["seconds_per_point_pass"] = {"cuda_fp64": t64s / points_passes, "cuda_c64": t32 / points_passes,
                                     "reference_cuda_fp64": tref3 / points_passes if tref3 else None,
                                     "reference_value_cuda": 4.6e-8,
                                     "workload": "microlens 512^2 x 400 slabs x 6 iterations, run only"}
    del r32, r64, p
    # 2: Born fluctuation at full size, 4096 points, 2000 slabs, 6 iterations, TE
    p = workloads.born2d(polarization="te")
    r32, t32 = timed(lambda: _core.CudaSolver(*p.core_args(), device, fluctuation=p.fluctuation,
                                              precision=32).run(p.field, p.iterations, []))
    r64, t64s = timed(lambda: _core.CudaSolver(*p.core_args(), device,
                                               fluctuation=p.fluctuation).run(p.field, p.iterations, []))
    out["born2d"] = {"c64_s": t32, "fp64_s": t64s,
                     "l2_err_transmitted": _rel(r32["transmitted"], r64["transmitted"]),
                     "l2_err_reflected": _rel(r32["reflected"], r64["reflected"]),
                     "workload": "4096 points, 2000 slabs, delta-n (std 0.01, 0.5 um) on every slab, "
                                 "10 deg plane wave, 6 iterations, TE; set-up included"}
    return out


def run_plane3d(n: int) -> None:
    """A small 3D case for profiling the slab-step kernels (k_cols_step, k_rows_select)."""
    from bwpm_b200 import _core, workloads

    p = workloads.microlens3d(n=n, nz=24, iterations=1)
    s = _core.CudaSolver(*p.core_args(), 0, precision=32)
    t0 = time.perf_counter()
    s.run(p.field, 1, [])
    print(json.dumps({"plane3d": n, "run_s": time.perf_counter() - t0, **s.stats()}), flush=True)


def prm_wl(prm: dict) -> float:
    return float(prm["wl"])


def _peak_source() -> str:
    """Where the HBM peak came from: the measured file of this pool, or the fallback figure."""
    return "measured" if (ROOT / "MEASURED_PEAKS.json").exists() else "fallback (6.65 TB/s)"


def _peak(key: str) -> float:
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())[key])
    except Exception:  # noqa: BLE001
        return {"hbm_gbs": 6650.0}.get(key, float("nan"))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--fp64-sample", type=int, default=6)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="instances per step of the CPU reference (default: 3 per host core)")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream measurement")
    ap.add_argument("--no-configs", action="store_true", help="skip the slab, Born and microlens workloads")
    ap.add_argument("--served-fp64", type=int, default=16, help="FP64 sample of the served stream")
    ap.add_argument("--variants", type=str, default="",
                    help="profiling only: NY:VARIANT,... forces kernel variants (no autotuning)")
    ap.add_argument("--reduced", type=str, default="",
                    help="profiling only: COUNT,NZ_MAX,ITERATIONS[,NY] (first COUNT solves, chains "
                         "capped, optionally all of length NY); skips the FP64, served and CPU "
                         "comparisons")
    ap.add_argument("--plane3d", type=int, default=0,
                    help="profiling only: one complex64 3D microlens solve of N^2 points, 24 slabs, "
                         "1 iteration (the 3D slab-step kernels), then exit")
    args = ap.parse_args()
    if args.plane3d:
        run_plane3d(args.plane3d)
        return
    if args.reduced:
        vals = [int(v) for v in args.reduced.split(",")]
        REDUCED.update(count=vals[0], nz_max=vals[1], iterations=vals[2],
                       ny=vals[3] if len(vals) > 3 else None)
        args.no_cpu = True
        args.no_served = True
        args.no_configs = True
        args.fp64_sample = 0
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
