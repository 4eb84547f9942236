"""Benchmark: kNN sources/s, 4M points, k = 32, one B200.

Workload: the bimodal triclinic configuration (4,000,000 seeded synthetic
points in the sheared cell a=(L,0,0), b=(0.3L,0.95L,0), c=(0.1L,0.2L,0.97L),
density 0.1 on one half and 0.005 on the other, 1 % of points on bin
faces, 0.5 % exact duplicates; k = 32; cell_hint = 3.0; no mask).

One step = one full search of that frame (fold, bin, scan, placement, walk,
replay) with inputs resident in HBM. The L2 (126 MB) is flushed between
timed steps by writing a 256 MB buffer; each step also writes 1.5 GB of
output rows.

--impl reference times the reference CPU walk (the C++ restatement of
src/knearest.rs in oracle/, on every host thread): each step is the fold,
bin and linked lists over all points plus the walk of a quarter of the
sources (every 4th, rotating), timed as it runs.

Beside the headline, the default run reports: the rooflines of the walk
(reference candidate pairs per second against the FP32-issue bound) and of
the prep (fold, bin, scan, placement against HBM); the network against the
best constant shell proposal on the same select walk; the batched-frames
configuration (256 frames in one graph-replayed call, and end to end through
lc_knearest_batch); the reference CPU walk on all host threads and on one;
the reference's gpulite GPU path; and a parity sample against the oracle.

Under torchrun each rank runs its own frame on its own GPU (no collective on
the data path; weak scaling); timings are the max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import platform
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "kNN sources/s, 4M pts k=32, 1 B200: FP32+learned vs plain walk, exact indices"
MODE_NAMES = {0: "plain_f64", 1: "fast_f32", 2: "learned", 3: "replay"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=60)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", type=int, default=-1, help="walk mode; -1 = best available")
    p.add_argument("--n", type=int, default=4_000_000)
    p.add_argument("--k", type=int, default=32)
    p.add_argument("--tpp", type=int, default=0,
                   help="threads per source of the headline walk: 32 or 1; 0 lets the "
                        "autotuner pick")
    p.add_argument("--plain-tpp", type=int, default=0,
                   help="the same for the plain FP64 walk timed beside it")
    p.add_argument("--walk-shape", default="",
                   help="W,G: force the select walk's warps per block and work grab "
                        "(the autotuner's choice otherwise); for profiling one shape")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-sweep", action="store_true",
                   help="skip the network-vs-constant-proposal sweep")
    p.add_argument("--no-c3", action="store_true", help="skip the batched-frames block")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-gpulite", action="store_true",
                   help="skip the reference's gpulite GPU path timed beside the headline")
    p.add_argument("--gpulite-child", action="store_true", help=argparse.SUPPRESS)
    p.add_argument("--workload", default="c2", choices=["c2", "c3"],
                   help="c2: the 4M bimodal frame (headline); c3: 256 frames of uneven n, "
                        "cell, k and mask in one batched call")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(x: float, device: str) -> float:
    """The largest x over the ranks of the default process group (x itself
    without one): every multi-GPU time is the slowest rank's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, max_ms: float, world: int) -> float:
    """Units of all ranks per second over the slowest rank's time (weak
    scaling: every rank searches its own frame)."""
    return world * units_per_rank * steps / (max_ms / 1000.0)


def workload_name(n, k):
    """Name of the bimodal workload of n points and k neighbours."""
    return "bimodal_triclinic_4M_k32" if (n, k) == (4_000_000, 32) else f"bimodal_triclinic_n{n}_k{k}"


def workload(n, k, seed):
    from linkcell_b200 import workloads as W
    return W.bimodal_triclinic(n=n, seed=seed, k=k)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,utilization.gpu")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        load = [r for r in self.rows if (num(r[7]) or 0) > 0] or self.rows
        sm = [num(r[0]) for r in load if num(r[0]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for name, v in zip(names, r[3:7]):
                if v.strip().lower() in ("active", "1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": num(self.rows[0][1]), "reasons": sorted(reasons),
                "samples": len(self.rows), "power_w_max": max(num(r[2]) or 0 for r in self.rows)}


def host_info():
    """The host the CPU figures come from: name, CPU model, logical cores."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"host": platform.node(), "cpu_model": model, "logical_cores": os.cpu_count()}


def _sampled_rate(O, w, threads, seconds_target):
    """The reference walk on `threads` threads: fold + bin + lists over all
    points, then the walk of an evenly strided sample of sources sized to
    about seconds_target; sources/s of the whole frame with the walk time
    scaled from the sample."""
    n = w["xyz"].shape[0]
    probe = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"], first=0,
                          stride=max(1, n // 4000), count=4000, threads=threads)
    per_src = probe["walk_s"] / max(1, probe["walked"])
    count = int(max(4000, min(n, seconds_target / max(per_src, 1e-9))))
    stride = max(1, n // count)
    r = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"], first=0,
                      stride=stride, count=count, threads=threads)
    est_total = r["prep_s"] + r["walk_s"] * (n / max(1, r["walked"]))
    return n / est_total, r, stride


def cpu_baseline(w, seconds_target=15.0):
    """The reference walk restated in oracle/ on all host threads, and on one
    thread, each on a bounded sample of sources (scaled to sources/s of the
    whole frame; the sample is stated)."""
    from oracle import oracle as O
    O.build()
    n = w["xyz"].shape[0]
    threads = os.cpu_count() or 1
    v, r, stride = _sampled_rate(O, w, threads, seconds_target)
    v1, r1, stride1 = _sampled_rate(O, w, 1, seconds_target / 3.0)
    return {"value": v, "unit": "sources/s", "cores": threads, "kind": "port",
            "sample": (f"fold+bin+lists over all {n} points ({r['prep_s']:.2f} s) plus the walk of "
                       f"{r['walked']} sources (every {stride}-th, {r['walk_s']:.2f} s), the walk "
                       f"time scaled to all sources"),
            "single_core": {"value": v1, "unit": "sources/s", "cores": 1,
                            "sample": (f"the same on one thread: prep {r1['prep_s']:.2f} s, walk of "
                                       f"{r1['walked']} sources (every {stride1}-th, "
                                       f"{r1['walk_s']:.2f} s)")},
            **host_info()}


def parity_sample(w, nn, d2, count=20000):
    """The oracle as the checker, beside the CPU baseline: the rows of a seeded
    sample of sources from the timed search against the reference walk's
    (oracle.knearest_subset): rows whose indices differ, and the largest
    relative dist2 difference."""
    import torch
    from oracle import oracle as O
    O.build()
    n = w["xyz"].shape[0]
    src = np.sort(np.random.default_rng(7).choice(n, size=min(count, n), replace=False))
    want_nn, want_d2, visits = O.knearest_subset(w["xyz"], w["cell"], w["k"], src,
                                                 mask=w.get("mask"), cell_hint=w["cell_hint"],
                                                 threads=os.cpu_count() or 1, with_visits=True)
    idx = torch.as_tensor(src, device=nn.device)
    got_nn, got_d2 = nn[idx].cpu().numpy(), d2[idx].cpu().numpy()
    bad_rows = int((got_nn != want_nn).any(axis=1).sum())
    finite = np.isfinite(want_d2)
    both_nan = ~finite & np.isnan(got_d2)
    rel = np.abs(got_d2[finite] - want_d2[finite]) / np.maximum(np.abs(want_d2[finite]), 1e-300)
    return {"sources": int(src.size), "index_mismatch_rows": bad_rows,
            "dist2_max_rel_err": float(rel.max()) if rel.size else 0.0,
            "dist2_nan_agree": bool(both_nan.sum() == (~finite).sum()),
            "ref_pairs_per_source": float(visits.mean()),
            "checker": "oracle reference walk (knearest_subset), seeded sample of the timed rows"}


GPULITE_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_gpulite.so")
GPULITE_K = 16            # the gpulite path supports k <= 16 (src/gpu/knearest.cpp:23)
GPULITE_CELLS = 262144    # ... and at most this many cells (src/gpu/knearest.cpp:24)


def gpulite_hint(cell, k_cap=GPULITE_CELLS):
    """The smallest cell edge (3.0 and up, in steps of 0.05) whose mesh of
    the given cell stays within the gpulite path's cell cap."""
    h = np.asarray(cell, dtype=np.float64)
    a, b, c = h[0], h[1], h[2]
    det = abs(float(np.dot(a, np.cross(b, c))))
    widths = [det / np.linalg.norm(np.cross(b, c)), det / np.linalg.norm(np.cross(c, a)),
              det / np.linalg.norm(np.cross(a, b))]
    edge = 3.0
    while np.prod([max(1, int(np.floor(wd / edge))) for wd in widths]) > k_cap:
        edge = round(edge + 0.05, 2)
    return edge


def gpulite_child(args):
    """Child process of the gpulite leg: the reference's own gpulite GPU path
    (src/gpu/knearest.cpp + capi.cpp, built from the reference sources into
    oracle/_ref by oracle/build_ref.sh) timed through its C ABI on the same
    points as the headline, at k = 16 and the smallest cell edge its cell cap
    allows. Only that library is loaded here (it exports the same lc_gpu_*
    names as ours). Prints one JSON line."""
    import torch
    torch.cuda.set_device(0)
    lib = ctypes.CDLL(GPULITE_LIB)
    vp, sz, d, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_int
    lib.lc_gpu_workspace_new.restype = vp
    lib.lc_gpu_workspace_free.argtypes = [vp]
    lib.lc_gpu_last_error.restype = ctypes.c_char_p
    lib.lc_gpu_knearest_many.argtypes = [vp, vp, sz, sz, vp, sz, vp, d, vp, vp, i]
    w = workload(args.n, args.k, seed=2)
    n = w["xyz"].shape[0]
    hint = gpulite_hint(w["cell"])
    rows = np.asarray(w["cell"], dtype=np.float64).reshape(-1)
    cell = (ctypes.c_double * 12)(*[float(v) for v in rows], 0.0, 0.0, 0.0)
    x = torch.as_tensor(w["xyz"], device="cuda")
    nn = torch.empty((n, GPULITE_K), dtype=torch.int32, device="cuda")
    d2 = torch.empty((n, GPULITE_K), dtype=torch.float64, device="cuda")
    ws = lib.lc_gpu_workspace_new()
    if not ws:
        print(json.dumps({"unavailable": (lib.lc_gpu_last_error() or b"").decode()}))
        return

    def step():
        rc = lib.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), GPULITE_K, None,
                                      hint, nn.data_ptr(), d2.data_ptr(), 1)
        if rc != 0:
            raise RuntimeError((lib.lc_gpu_last_error() or b"").decode())
    torch.cuda.synchronize()
    for _ in range(max(2, args.warmup)):  # the first call compiles the kernels (nvrtc)
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    lib.lc_gpu_workspace_free(ws)
    ms = 1000.0 * statistics.median(times)
    print(json.dumps({"value": n / (ms / 1000.0), "ms_per_step": ms, "k": GPULITE_K,
                      "cell_hint": hint, "n": n}))


def gpulite_leg(args, L, ws, x, n):
    """The reference's gpulite GPU path, timed in a child process, and ours
    on the same configuration (k = 16, the same cell edge), both as
    synchronous calls with inputs resident on the device, median wall time."""
    import torch
    if not os.path.exists(GPULITE_LIB):
        return {"unavailable": "oracle/_ref/libref_gpulite.so not built (no reference sources)"}
    steps = 5
    cmd = [sys.executable, os.path.abspath(__file__), "--gpulite-child", "--n", str(args.n),
           "--k", str(args.k), "--steps", str(steps), "--warmup", "2"]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"unavailable": "gpulite child did not finish in 900 s"}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        tail = (r.stderr.strip().splitlines() or ["no output"])[-1]
        return {"unavailable": f"gpulite child failed: {tail[:200]}"}
    ref = json.loads(lines[-1])
    if "unavailable" in ref:
        return ref
    from linkcell_b200 import _capi
    from linkcell_b200 import _cell_struct
    w = workload(args.n, args.k, seed=2)
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    nn = torch.empty((n, GPULITE_K), dtype=torch.int32, device="cuda")
    d2 = torch.empty((n, GPULITE_K), dtype=torch.float64, device="cuda")

    def step():
        rc = L.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), GPULITE_K, None,
                                    ref["cell_hint"], nn.data_ptr(), d2.data_ptr(), 1)
        assert rc == 0, _capi.gpu_error()
    for _ in range(3):
        step()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    ours_ms = 1000.0 * statistics.median(times)
    del nn, d2
    return {"value": ref["value"], "unit": "sources/s", "ms_per_step": ref["ms_per_step"],
            "config": (f"the headline's {n} points at k = {GPULITE_K} and cell_hint "
                       f"{ref['cell_hint']} (the gpulite path takes k <= 16 and at most "
                       f"{GPULITE_CELLS} cells, so it cannot run the k = 32 headline)"),
            "timer": "host wall clock around a synchronous call, median of 5",
            "kind": "reference gpulite (src/gpu/knearest.cpp, nvrtc-compiled at run time)",
            "ours_same_config": {"value": n / (ours_ms / 1000.0), "ms_per_step": ours_ms,
                                 "mode": "learned"}}


REF_PARTS = 4  # a reference step walks every REF_PARTS-th source


def run_reference(args):
    """The reference CPU walk (the oracle's restatement of src/knearest.rs,
    kind "port": the image has no Rust toolchain) on all host threads. Each
    step is timed as it runs: fold + bin + linked lists over all points, then
    the walk of every 4th source (offset rotating by step), so a step walks a
    quarter of the frame's sources; value = sources walked / step time."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    w = workload(args.n, args.k, seed=2)
    from oracle import oracle as O
    O.build()
    n = w["xyz"].shape[0]
    threads = os.cpu_count() or 1
    count = (n + REF_PARTS - 1) // REF_PARTS
    secs, walked = [], []
    for step in range(args.warmup + args.steps):
        r = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"],
                          first=step % REF_PARTS, stride=REF_PARTS, count=count, threads=threads)
        if step >= args.warmup:
            secs.append(r["prep_s"] + r["walk_s"])
            walked.append(r["walked"])
    v = sum(walked) / sum(secs)
    ms = 1000.0 * sum(secs) / len(secs)
    out = {"metric": METRIC, "value": v, "unit": "sources/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": workload_name(n, args.k), "n": n, "k": args.k,
                      "cell_hint": 3.0, "l2": "n/a (CPU)"},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "sources/s", "cores": threads, "kind": "port",
                            "sample": (f"each step: fold+bin+lists over all {n} points, then the "
                                       f"walk of every {REF_PARTS}th source ({walked[0]} "
                                       f"sources), timed as it runs"),
                            **host_info()},
           "e2e": {"value": v, "unit": "sources/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


COUNTER_NAMES = ["pairs", "inserts", "replays", "shells", "pruned", "reranks", "prop_under",
                 "prop_over", "prop_exact", "revisited", "fallback"]


def prep_roofline(frame_rows, n, prep_ms, peak):
    """Fold, bin, scan and placement against HBM: the design-independent
    minimum per search (read the coordinates, write the cell-sorted FP64
    coordinates and the point index, count and offset per cell) over the
    measured prep time, and the DRAM traffic of those kernels from the
    committed ncu summary, where there is one."""
    from linkcell_b200 import workloads as W
    cells = int(np.prod(W.bins_of(np.asarray(frame_rows, dtype=np.float64))))
    algo = n * (24 + 24 + 4) + 8 * (cells + 1)
    achieved = algo / (prep_ms / 1000.0) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "prep_bimodal_4M_traffic.txt")
    if os.path.exists(tpath) and n == 4_000_000:
        for line in open(tpath):
            if line.startswith("traffic_bytes_per_search:"):
                traffic = float(line.split(":")[1])
    return {"bound": "hbm", "unit": "GB/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "algorithmic_bytes": algo,
            "bytes_per_point": algo / n, "ms": prep_ms, "traffic": traffic,
            "traffic_over_algorithmic": None if traffic is None else traffic / algo,
            "kernels": "k_fold_bin, k_scan_cells, k_place_slots, k_place_records"}


def walk_roofline(ref_pairs, walk_ms, f_sm_mhz, sms):
    """The walk in candidate-pair evaluations as the reference visits them
    (its heap pushes: every occupant of every cell of shells 1..R*, minus the
    source) per second, against the FP32-issue bound of about 8 FP32
    instructions per pair: SMs x 128 lanes x f_SM / 8."""
    achieved = ref_pairs / (walk_ms / 1000.0)
    peak = sms * 128 * f_sm_mhz * 1e6 / 8.0
    return {"bound": "fp32_issue", "unit": "pair-evals/s", "achieved": achieved, "peak": peak,
            "frac": achieved / peak, "ref_pairs": ref_pairs, "walk_ms": walk_ms,
            "f_sm_mhz": f_sm_mhz, "sms": sms}


def step_roofline(sources_per_s, prep_bytes_per_point, k, ref_pairs_per_source, peak_gbs, f_sm_mhz,
                  sms):
    """The whole search in sources/s against the slower of two bounds: HBM
    for the prep's minimum plus the output row ((57.2 + 12 k) B per source on
    this workload) and the FP32 issue bound for the reference's mean pairs per
    source (SMs x 128 lanes x f_SM / 8 pair-evaluations/s)."""
    hbm = peak_gbs * 1e9 / (prep_bytes_per_point + 12.0 * k)
    walk = sms * 128 * f_sm_mhz * 1e6 / 8.0 / ref_pairs_per_source
    peak = min(hbm, walk)
    return {"bound": "hbm" if hbm <= walk else "fp32_issue", "unit": "sources/s",
            "achieved": sources_per_s, "peak": peak, "frac": sources_per_s / peak,
            "hbm_bound": hbm, "walk_bound": walk,
            "bytes_per_source": prep_bytes_per_point + 12.0 * k,
            "ref_pairs_per_source": ref_pairs_per_source}


def run_ours(args):
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    from linkcell_b200 import _capi
    from linkcell_b200 import build as B
    from linkcell_b200 import _cell_struct
    B.build()
    L = _capi.load()
    w = workload(args.n, args.k, seed=2 + rank)
    n, k = w["xyz"].shape[0], w["k"]
    cell = _cell_struct(np.asarray(w["cell"], dtype=np.float64))
    x = torch.as_tensor(w["xyz"], device="cuda")
    nn = torch.empty((n, k), dtype=torch.int32, device="cuda")
    d2 = torch.empty((n, k), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    ws = L.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    stream = ctypes.c_void_p(L.lc_gpu_queue(ws))
    tstream = torch.cuda.ExternalStream(stream.value)

    def step():
        rc = L.lc_gpu_knearest_many(ws, x.data_ptr(), n, 1, ctypes.byref(cell), k, None, 3.0,
                                    nn.data_ptr(), d2.data_ptr(), 0)
        assert rc == 0, _capi.gpu_error()

    model_info = None
    if (args.mode if args.mode >= 0 else 2) == 2:
        from linkcell_b200 import learn
        if os.path.exists(learn.MODEL_PATH):
            learn.attach(ws)
            _, tau, meta = learn.load()
            model_info = {"path": os.path.relpath(learn.MODEL_PATH, ROOT), "tau": tau, "trained": meta}

    def time_mode(mode, steps, warmup, tpp, shell=0):
        """steps timed searches of one configuration (shell > 0: that shell
        proposed for every source instead of the network's proposals), then
        one untimed search that counts the walk statistics."""
        assert L.lc_gpu_set_mode(ws, mode) == 0
        assert L.lc_gpu_set_tpp(ws, tpp) == 0  # 0: the autotuner's choice
        if args.walk_shape:
            wwarps, wgrab = (int(v) for v in args.walk_shape.split(","))
            assert L.lc_gpu_set_walk_shape(ws, wwarps, wgrab) == 0
        assert L.lc_gpu_set_proposal(ws, shell) == 0
        for _ in range(warmup):
            step()
            L.lc_gpu_wait(ws)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        walk_ms, prep_ms, replay_ms, prop_ms = [], [], [], []
        for s in range(steps):
            with torch.cuda.stream(tstream):
                flush.fill_(s & 0xFF)  # L2 flush between timed steps, outside the events
                ev[s][0].record(tstream)
            step()
            with torch.cuda.stream(tstream):
                ev[s][1].record(tstream)
            L.lc_gpu_wait(ws)
            pp, pq, pw, pr = (ctypes.c_double(), ctypes.c_double(), ctypes.c_double(),
                              ctypes.c_double())
            L.lc_gpu_phase_times4(ws, ctypes.byref(pp), ctypes.byref(pq), ctypes.byref(pw),
                                  ctypes.byref(pr))
            walk_ms.append(pw.value)  # the walk kernel alone
            prop_ms.append(pq.value)
            prep_ms.append(pp.value)
            replay_ms.append(pr.value)
        torch.cuda.synchronize()
        # the walk statistics cost time: one more search, untimed, counts them
        assert L.lc_gpu_set_stats(ws, 1) == 0
        step()
        L.lc_gpu_wait(ws)
        assert L.lc_gpu_set_stats(ws, 0) == 0
        buf = (ctypes.c_longlong * 16)()
        L.lc_gpu_stats(ws, buf, 16, None)
        counters = {nm: int(buf[i]) for i, nm in enumerate(COUNTER_NAMES)}
        counters["tpp"] = int(L.lc_gpu_get_tpp(ws))  # walk design used (autotuned unless forced)
        shp = (ctypes.c_int * 3)()
        L.lc_gpu_walk_shape(ws, shp, None, 0)
        counters["shape"] = list(shp)
        assert L.lc_gpu_set_proposal(ws, 0) == 0
        total = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), "cuda")
        return {"total_ms": total, "ms": total / steps, "walk_ms": statistics.mean(walk_ms),
                "prep_ms": statistics.mean(prep_ms), "replay_ms": statistics.mean(replay_ms),
                "propose_ms": statistics.mean(prop_ms), "counters": counters}

    best_mode = args.mode if args.mode >= 0 else 2
    # plain FP64 walk (the 2x denominator), then the headline mode
    sampler = ClockSampler(dev)
    sampler.start()  # clocks over both timed regions
    time.sleep(0.3)  # nvidia-smi start-up
    plain_steps = max(3, args.steps // 2)
    plain = time_mode(0, plain_steps, args.warmup, args.plain_tpp)
    head = time_mode(best_mode, args.steps, args.warmup, args.tpp)
    sampler.stop()
    clocks = sampler.summary()
    ms_per_step = head["ms"]
    value = whole_job_rate(n, args.steps, head["total_ms"], world)
    plain_value = whole_job_rate(n, plain_steps, plain["total_ms"], world)

    # roofline of the dominant kernel (the walk): algorithmic bytes per launch
    peak, peak_kind = measured_peaks()
    # per source: FP32 record 16 B + FP64 coordinates 24 B + index and cell 8 B read,
    # the output row (i32 + f64 per slot) written
    walk_bytes = n * (48 + 12 * k)
    walk_avg_ms = head["walk_ms"]
    achieved = walk_bytes / (walk_avg_ms / 1000.0) / 1e9
    traffic = None
    tname = "select_walk" if best_mode == 2 else "walk"
    tpath = os.path.join(ROOT, "profiles", f"{tname}_bimodal_4M_k32_traffic.txt")
    if os.path.exists(tpath) and (n, k) == (4_000_000, 32):
        for line in open(tpath):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":")[1])
    f_sm = clocks.get("sm_mhz") or 1965.0
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "k_select_walk" if best_mode == 2 else "walk",
                "algorithmic_bytes_per_source": 48 + 12 * k,
                # the plain FP64 walk visits exactly the reference's pairs (its
                # counter equals the oracle's heap pushes: 348.65 per source here)
                "walk": walk_roofline(float(plain["counters"]["pairs"]), walk_avg_ms, f_sm, sms),
                "prep": prep_roofline(w["cell"], n, head["prep_ms"], peak)}
    roofline["step"] = step_roofline(value, roofline["prep"]["bytes_per_point"], k,
                                     float(plain["counters"]["pairs"]) / n, peak, f_sm, sms)

    # the network against one constant shell for every source, same select walk
    lvc = None
    if best_mode == 2 and model_info is not None and not args.no_sweep:
        sweep = []
        for shell in range(1, 7):
            r = time_mode(2, 5, 1, args.tpp, shell=shell)
            sweep.append({"shell": shell, "ms": r["ms"], "walk_ms": r["walk_ms"],
                          "replay_ms": r["replay_ms"], **r["counters"]})
        best = min(sweep, key=lambda e: e["ms"])
        lvc = {"network": {"ms": head["ms"], "walk_ms": head["walk_ms"],
                           "propose_ms": head["propose_ms"], "replay_ms": head["replay_ms"],
                           **head["counters"]},
               "best_constant": best, "constant_sweep": sweep,
               "speedup_network_vs_best_constant": best["ms"] / head["ms"]}

    # end to end through the host C ABI with pinned buffers
    e2e = None
    if not args.no_e2e:
        hx = torch.as_tensor(w["xyz"]).pin_memory()
        hnn = torch.empty((n, k), dtype=torch.int32).pin_memory()
        hd2 = torch.empty((n, k), dtype=torch.float64).pin_memory()
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        # the host ABI walks with the library's default mode; select the headline mode
        os.environ["LINKCELL_MODE"] = str(best_mode)
        if args.tpp:
            os.environ["LINKCELL_TPP"] = str(args.tpp)

        def host_step():
            rc = L.lc_knearest_d2(ctypes.cast(hx.data_ptr(), dp), n, ctypes.byref(cell), k, None, 3.0,
                                  ctypes.cast(hnn.data_ptr(), ip), ctypes.cast(hd2.data_ptr(), dp))
            assert rc == 0, _capi.cpu_error()
        for _ in range(args.warmup):
            host_step()
        times = []
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            host_step()
            times.append(time.perf_counter() - t0)
        tot = max_over_ranks(sum(times), "cuda")
        e2e = {"value": whole_job_rate(n, args.steps, 1000.0 * tot, world), "unit": "sources/s",
               "h2d_bytes_per_step": n * 24, "d2h_bytes_per_step": n * k * 12,
               "ms_per_step": 1000.0 * tot / args.steps, "timer": "host wall clock around the call"}
        del hx, hnn, hd2

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, args.cpu_seconds)
        parity = parity_sample(w, nn, d2)
    gpulite = None
    if rank == 0 and world == 1 and not args.no_gpulite:
        assert L.lc_gpu_set_mode(ws, best_mode) == 0
        gpulite = gpulite_leg(args, L, ws, x, n)
    L.lc_gpu_workspace_free(ws)
    del x, nn, d2
    torch.cuda.empty_cache()
    c3 = None
    if rank == 0 and world == 1 and not args.no_c3:
        c3 = c3_block(args, max(5, args.steps // 2), world, flush)

    # our kernels per step: fold, scan, slots, records, walk, replay; the learned
    # mode adds the proposal network and the per-source proposal gather
    launches_per_step = 6 + (2 if (best_mode == 2 and model_info is not None) else 0)
    out = {"metric": METRIC, "value": value, "unit": "sources/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": workload_name(n, k), "n": n, "k": k, "cell_hint": 3.0,
                      "mode": MODE_NAMES[best_mode], "tpp": head["counters"]["tpp"],
                      "walk_shape": head["counters"]["shape"],
                      "tpp_source": "forced" if args.tpp else "autotuned",
                      "parallelism": f"replicas x{world}",
                      "l2": "flushed between timed steps (256 MB write)"},
           "roofline": roofline, "cpu_baseline": cpu, "gpulite_baseline": gpulite, "e2e": e2e,
           "parity_sample": parity,
           "gpu_launches": launches_per_step * args.steps, "clocks": clocks,
           "plain_fp64": {"value": plain_value, "unit": "sources/s", "walk_ms": plain["walk_ms"],
                          "tpp": plain["counters"]["tpp"]},
           "speedup_vs_plain": value / plain_value, "walk_ms": walk_avg_ms,
           "prep_ms": head["prep_ms"], "replay_ms": head["replay_ms"],
           "propose_ms": head["propose_ms"],
           "walk_stats_last_step": {nm: head["counters"][nm] for nm in COUNTER_NAMES},
           "learned_vs_constant": lvc, "c3": c3, "model": model_info,
           "plain_walk_stats_last_step": {nm: plain["counters"][nm] for nm in COUNTER_NAMES}}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def c3_block(args, steps, world, flush):
    """The batched-frames configuration: 256 frames of their own sheared
    cells, densities, k in {4, 8, 16, 32} and masks
    (linkcell_b200.workloads.frames_batch, seed 3) searched by one
    lc_gpu_knearest_batch call per step, the launch sequence captured once
    in a CUDA graph and replayed; value = active sources of all frames per
    second (device time), beside the plain FP64 walk; e2e is the same batch
    through lc_knearest_batch with host buffers: the copies of the
    coordinates and mask in and of the rows out."""
    import torch
    from linkcell_b200 import _capi, _cell_struct, learn, workloads as W
    L = _capi.load()
    rank = dist_env()[1]
    frames = W.frames_batch(256, seed=3 + rank)
    arr = (_capi.LcFrame * len(frames))()
    total_out, moff, active = 0, 0, 0
    for f, fr in enumerate(frames):
        arr[f].n, arr[f].k = fr["n"], fr["k"]
        arr[f].cell = _cell_struct(np.asarray(fr["cell"], dtype=np.float64))
        arr[f].cell_hint = 3.0
        arr[f].mask_offset = moff
        moff += fr["n"]
        total_out += fr["n"] * fr["k"]
        active += int(fr["mask"].sum())
    xyz_h = np.concatenate([fr["xyz"] for fr in frames])
    mask_h = np.concatenate([fr["mask"] for fr in frames]).astype(np.int32)
    x = torch.as_tensor(xyz_h, device="cuda")
    m = torch.as_tensor(mask_h, device="cuda")
    nn = torch.empty(total_out, dtype=torch.int32, device="cuda")
    d2 = torch.empty(total_out, dtype=torch.float64, device="cuda")
    ws = L.lc_gpu_workspace_new()
    assert ws, _capi.gpu_error()
    learn.attach(ws)
    assert L.lc_gpu_set_graph(ws, 1) == 0
    if args.tpp:
        assert L.lc_gpu_set_tpp(ws, args.tpp) == 0
    tstream = torch.cuda.ExternalStream(ctypes.c_void_p(L.lc_gpu_queue(ws)).value)

    def step():
        rc = L.lc_gpu_knearest_batch(ws, x.data_ptr(), arr, len(frames), m.data_ptr(),
                                     nn.data_ptr(), d2.data_ptr(), 0)
        assert rc == 0, _capi.gpu_error()

    def time_mode(mode, steps):
        assert L.lc_gpu_set_mode(ws, mode) == 0
        for _ in range(args.warmup):
            step()
            L.lc_gpu_wait(ws)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        for i in range(steps):
            with torch.cuda.stream(tstream):
                flush.fill_(i & 0xFF)
                ev[i][0].record(tstream)
            step()
            with torch.cuda.stream(tstream):
                ev[i][1].record(tstream)
        L.lc_gpu_wait(ws)
        torch.cuda.synchronize()
        return max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), "cuda")

    plain_ms = time_mode(0, max(3, steps // 2))
    total_ms = time_mode(2, steps)
    value = whole_job_rate(active, steps, total_ms, world)
    plain_value = whole_job_rate(active, max(3, steps // 2), plain_ms, world)
    captures = int(L.lc_gpu_graph_captures(ws))
    shape = (ctypes.c_int * 3)()
    trials = (ctypes.c_int * 48)()
    ntrial = L.lc_gpu_walk_shape(ws, shape, trials, 16)

    # end to end through lc_knearest_batch: the same batch from host memory
    # (page-locked), rows back into page-locked buffers, which the library
    # copies in row ranges while the rest of the batch is searched
    xh = torch.as_tensor(xyz_h).pin_memory()
    mh = torch.as_tensor(mask_h).pin_memory()
    nnh = torch.empty(total_out, dtype=torch.int32).pin_memory()
    d2h = torch.empty(total_out, dtype=torch.float64).pin_memory()
    os.environ["LINKCELL_MODE"] = "2"  # the host ABI's workspace: the learned walk

    def host_step():
        rc = L.lc_knearest_batch(xh.data_ptr(), arr, len(frames), mh.data_ptr(), nnh.data_ptr(),
                                 d2h.data_ptr())
        assert rc == 0, _capi.cpu_error()

    times = []
    for i in range(args.warmup + steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        host_step()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(times), "cuda")
    ks = sorted({fr["k"] for fr in frames})
    out = {"metric": "kNN sources/s, 256 frames of uneven n, cell, k and mask in one call, "
                     "exact indices",
           "value": value, "unit": "sources/s", "steps": steps, "ms_per_step": total_ms / steps,
           "config": {"workload": "batched_256_frames_seed3", "frames": len(frames),
                      "points": int(moff), "active_sources": active, "k": ks, "mode": "learned",
                      "graph": True, "graph_captures": captures,
                      "walk_shape": {"tpp": shape[0], "warps_per_block": shape[1],
                                     "grab": shape[2], "source": "autotuned",
                                     "candidates_timed": [list(trials[3 * i:3 * i + 3])
                                                          for i in range(ntrial)]},
                      "l2": "flushed between timed steps (256 MB write)"},
           "e2e": {"value": whole_job_rate(active, steps, 1000.0 * e2e_s, world),
                   "unit": "sources/s", "h2d_bytes_per_step": int(xyz_h.nbytes + mask_h.nbytes),
                   "d2h_bytes_per_step": int(total_out * 12),
                   "ms_per_step": 1000.0 * e2e_s / steps,
                   "timer": "host wall clock around lc_knearest_batch with host buffers"},
           "plain_fp64": {"value": plain_value, "unit": "sources/s"},
           "speedup_vs_plain": value / plain_value}
    # the copies above ran on the workspace's stream: release every tensor
    # that recorded it before the stream goes away with the workspace
    torch.cuda.synchronize()
    del x, m, nn, d2, xh, mh, nnh, d2h
    L.lc_gpu_workspace_free(ws)
    return out


def run_c3(args):
    """--workload c3: the batched-frames block alone, as its own JSON line."""
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from linkcell_b200 import build as B
    B.build()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.3)
    blk = c3_block(args, args.steps, world, flush)
    sampler.stop()
    out = {"metric": blk["metric"], "value": blk["value"], "unit": "sources/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": blk["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {**blk["config"], "parallelism": f"replicas x{world}"},
           "roofline": None, "cpu_baseline": None, "e2e": blk["e2e"], "gpu_launches": None,
           "clocks": sampler.summary(), "plain_fp64": blk["plain_fp64"],
           "speedup_vs_plain": blk["speedup_vs_plain"]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    args = parse()
    if args.gpulite_child:
        gpulite_child(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "c3":
        run_c3(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
