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
src/knearest.rs in oracle/, on every host thread) on a bounded sample of
sources of the same workload.

Under torchrun each rank runs its own frame on its own GPU (no collective on
the data path; weak scaling); timings are the max over ranks.
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
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
    p.add_argument("--no-e2e", action="store_true")
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


def cpu_baseline(w, seconds_target=15.0):
    """The reference walk restated in oracle/ on all host threads, on a bounded
    sample of sources; extrapolated to sources/s of the whole frame."""
    from oracle import oracle as O
    O.build()
    n = w["xyz"].shape[0]
    threads = os.cpu_count() or 1
    probe = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"], first=0,
                          stride=max(1, n // 20000), count=20000, threads=threads)
    per_src = probe["walk_s"] / max(1, probe["walked"])
    count = int(max(20000, min(n, seconds_target / max(per_src, 1e-9))))
    stride = max(1, n // count)
    r = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"], first=0,
                      stride=stride, count=count, threads=threads)
    est_total = r["prep_s"] + r["walk_s"] * (n / max(1, r["walked"]))
    return {"value": n / est_total, "unit": "sources/s", "cores": threads, "kind": "port",
            "sample": (f"fold+bin+lists over all {n} points ({r['prep_s']:.2f} s) plus the walk of "
                       f"{r['walked']} sources (every {stride}-th, {r['walk_s']:.2f} s), "
                       f"extrapolated to all sources")}


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
    want_nn, want_d2 = O.knearest_subset(w["xyz"], w["cell"], w["k"], src, mask=w.get("mask"),
                                         cell_hint=w["cell_hint"], threads=os.cpu_count() or 1)
    idx = torch.as_tensor(src, device=nn.device)
    got_nn, got_d2 = nn[idx].cpu().numpy(), d2[idx].cpu().numpy()
    bad_rows = int((got_nn != want_nn).any(axis=1).sum())
    finite = np.isfinite(want_d2)
    both_nan = ~finite & np.isnan(got_d2)
    rel = np.abs(got_d2[finite] - want_d2[finite]) / np.maximum(np.abs(want_d2[finite]), 1e-300)
    return {"sources": int(src.size), "index_mismatch_rows": bad_rows,
            "dist2_max_rel_err": float(rel.max()) if rel.size else 0.0,
            "dist2_nan_agree": bool(both_nan.sum() == (~finite).sum()),
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


def run_reference(args):
    world, rank, _ = dist_env()
    if rank != 0:
        return
    w = workload(args.n, args.k, seed=2)
    from oracle import oracle as O
    O.build()
    n = w["xyz"].shape[0]
    threads = os.cpu_count() or 1
    # bounded sample per step so the whole run stays within minutes
    count = int(os.environ.get("LINKCELL_REF_SAMPLE", "60000"))
    stride = max(1, n // count)
    vals = []
    for step in range(args.warmup + args.steps):
        r = O.time_sample(w["xyz"], w["cell"], w["k"], cell_hint=w["cell_hint"], first=step % stride,
                          stride=stride, count=count, threads=threads)
        if step >= args.warmup:
            vals.append(n / (r["prep_s"] + r["walk_s"] * (n / max(1, r["walked"]))))
    v = statistics.median(vals)
    ms = 1000.0 * n / v
    out = {"metric": METRIC, "value": v, "unit": "sources/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": workload_name(n, args.k), "n": n, "k": args.k,
                      "cell_hint": 3.0, "l2": "n/a (CPU)"},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "sources/s", "cores": threads, "kind": "port",
                            "sample": f"fold+bin over all {n} points plus the walk of every "
                                      f"{stride}-th source ({count} sources) per step, "
                                      "extrapolated to the whole frame"},
           "e2e": {"value": v, "unit": "sources/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


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

    def time_mode(mode, steps, warmup, tpp):
        assert L.lc_gpu_set_mode(ws, mode) == 0
        assert L.lc_gpu_set_tpp(ws, tpp) == 0  # 0: the autotuner's choice
        for _ in range(warmup):
            step()
            L.lc_gpu_wait(ws)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(steps)]
        walk_ms, prep_ms, replay_ms, prop_ms = [], [], [], []
        counters = None
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
        counters = list(buf)
        counters.append(int(L.lc_gpu_get_tpp(ws)))  # walk design used (autotuned unless forced)
        total = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), "cuda")
        return total, walk_ms, counters, prep_ms, replay_ms, prop_ms

    best_mode = args.mode if args.mode >= 0 else 2
    # plain FP64 walk (the 2x denominator), then the headline mode
    sampler = ClockSampler(dev)
    sampler.start()  # clocks over both timed regions
    time.sleep(0.3)  # nvidia-smi start-up
    plain_total, plain_walk, plain_cnt, _, _, _ = time_mode(0, max(3, args.steps // 2),
                                                            args.warmup, args.plain_tpp)
    total, walk_ms, cnt, prep_ms, replay_ms, prop_ms = time_mode(best_mode, args.steps,
                                                                 args.warmup, args.tpp)
    sampler.stop()
    ms_per_step = total / args.steps
    value = whole_job_rate(n, args.steps, total, world)
    plain_value = whole_job_rate(n, max(3, args.steps // 2), plain_total, world)

    # roofline of the dominant kernel (the walk): algorithmic bytes per launch
    peak, peak_kind = measured_peaks()
    # per source: FP32 record 16 B + FP64 coordinates 24 B + index and cell 8 B read,
    # the output row (i32 + f64 per slot) written
    walk_bytes = n * (48 + 12 * k)
    walk_avg_ms = statistics.mean(walk_ms)
    achieved = walk_bytes / (walk_avg_ms / 1000.0) / 1e9
    traffic = None
    tname = "select_walk" if best_mode == 2 else "walk"
    tpath = os.path.join(ROOT, "profiles", f"{tname}_bimodal_4M_k32_traffic.txt")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":")[1])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "peak_source": f"{peak_kind} hbm_gbs", "kernel": "k_select_walk" if best_mode == 2 else "walk",
                "algorithmic_bytes_per_source": 48 + 12 * k}

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

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, args.cpu_seconds)
        parity = parity_sample(w, nn, d2)
    gpulite = None
    if rank == 0 and world == 1 and not args.no_gpulite:
        assert L.lc_gpu_set_mode(ws, best_mode) == 0
        gpulite = gpulite_leg(args, L, ws, x, n)

    names = ["pairs", "inserts", "replays", "shells", "pruned", "reranks", "prop_under",
             "prop_over", "prop_exact", "revisited", "fallback"]
    walk_stats = {nm: cnt[i] for i, nm in enumerate(names)}  # an untimed step after the timing
    # our kernels per step: fold, scan, slots, records, walk, replay; the learned
    # mode adds the proposal network and the per-source proposal gather
    launches_per_step = 6 + (2 if (best_mode == 2 and model_info is not None) else 0)
    out = {"metric": METRIC, "value": value, "unit": "sources/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": workload_name(n, k), "n": n, "k": k, "cell_hint": 3.0,
                      "mode": MODE_NAMES[best_mode], "tpp": cnt[-1],
                      "tpp_source": "forced" if args.tpp else "autotuned",
                      "parallelism": f"replicas x{world}",
                      "l2": "flushed between timed steps (256 MB write)"},
           "roofline": roofline, "cpu_baseline": cpu, "gpulite_baseline": gpulite, "e2e": e2e,
           "parity_sample": parity,
           "gpu_launches": launches_per_step * args.steps, "clocks": sampler.summary(),
           "plain_fp64": {"value": plain_value, "unit": "sources/s",
                          "walk_ms": statistics.mean(plain_walk), "tpp": plain_cnt[-1]},
           "speedup_vs_plain": value / plain_value, "walk_ms": walk_avg_ms,
           "prep_ms": statistics.mean(prep_ms), "replay_ms": statistics.mean(replay_ms),
           "propose_ms": statistics.mean(prop_ms),
           "walk_stats_last_step": walk_stats, "model": model_info,
           "plain_walk_stats_last_step": {nm: plain_cnt[i] for i, nm in enumerate(names)}}
    if rank == 0:
        print(json.dumps(out), flush=True)
    L.lc_gpu_workspace_free(ws)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_c3(args):
    """C3: 256 frames of their own sheared cells, densities, k in {4, 8, 16, 32}
    and masks (linkcell_b200.workloads.frames_batch, seed 3) searched by one
    lc_gpu_knearest_batch call per step, the launch sequence captured once in
    a CUDA graph and replayed. value = active sources of all frames per
    second (device time); e2e is the same batch through lc_knearest_batch
    with host buffers: the copies of the coordinates and mask in and
    of the rows out."""
    import torch
    world, rank, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    from linkcell_b200 import _capi, _cell_struct, learn, workloads as W
    from linkcell_b200 import build as B
    B.build()
    L = _capi.load()
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
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
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

    sampler = ClockSampler(dev)
    sampler.start()
    time.sleep(0.3)
    plain_ms = time_mode(0, max(3, args.steps // 2))
    total_ms = time_mode(2, args.steps)
    sampler.stop()
    value = whole_job_rate(active, args.steps, total_ms, world)
    plain_value = whole_job_rate(active, max(3, args.steps // 2), plain_ms, world)
    captures = int(L.lc_gpu_graph_captures(ws))

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
    for i in range(args.warmup + args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        host_step()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(sum(times), "cuda")
    ks = sorted({fr["k"] for fr in frames})
    out = {"metric": "kNN sources/s, C3: 256 frames of uneven n, cell, k and mask, 1 B200, "
                     "exact indices",
           "value": value, "unit": "sources/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "c3_256_frames", "frames": len(frames), "points": int(moff),
                      "active_sources": active, "k": ks, "mode": "learned", "graph": True,
                      "graph_captures": captures, "parallelism": f"replicas x{world}",
                      "l2": "flushed between timed steps (256 MB write)"},
           "roofline": None, "cpu_baseline": None,
           "e2e": {"value": whole_job_rate(active, args.steps, 1000.0 * e2e_s, world),
                   "unit": "sources/s", "h2d_bytes_per_step": int(xyz_h.nbytes + mask_h.nbytes),
                   "d2h_bytes_per_step": int(total_out * 12),
                   "timer": "host wall clock around lc_knearest_batch with host buffers"},
           "gpu_launches": None, "clocks": sampler.summary(),
           "plain_fp64": {"value": plain_value, "unit": "sources/s"},
           "speedup_vs_plain": value / plain_value}
    if rank == 0:
        print(json.dumps(out), flush=True)
    # the copies above ran on the workspace's stream: release every tensor
    # that recorded it before the stream goes away with the workspace
    torch.cuda.synchronize()
    del x, m, nn, d2, xh, mh, nnh, d2h, flush
    L.lc_gpu_workspace_free(ws)
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
