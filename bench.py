#!/usr/bin/env python
"""Conjunction-screening benchmark: object-days/s screened on B200.

Workload (one "step" = one full screening call): 20,000 synthetic objects
over 1 day, 3-minute conjunction steps (480 steps), 5 km threshold.  The
polyjectory is built on the host from seeded elements by
``mizuba_b200.synth`` (1.9 GB of order-18 segments, larger than the 126 MB
L2, so no L2 flush is needed between timed steps).  Both forms are timed on
the same polyjectory: the plain FP64 form (bit-exact with the reference) and
the mixed form (FP32 broad phase on enclosing boxes, FP64 narrow phase); the
line reports that their conjunction sets are identical.

Our arm (default):
  value    object-days/s of the mixed form with the polyjectory resident in
           HBM, outputs left in HBM (device-side throughput, max over ranks);
           ``fp64_form`` holds the plain form's figures;
  e2e      the same metric through the C ABI from pinned host buffers: the
           polyjectory upload (H2D) and the copy of every output (D2H) are
           inside the timed region; the per-step arrays and trees stream to
           the host while the later stages compute (mzb_conjunctions_stream);
  roofline the dominant stage, from the library's CUDA-event stage timers;
  cpu_baseline the oracle port on this host's cores (rank 0, N = 1 only).
Reference arm (--impl reference): mizuba itself cannot be built here
(heyoka, TBB and Boost are absent), so the reference's CPU algorithm is
timed through the C++ restatement in oracle/ with all host threads.

Multi-GPU (torchrun): each rank screens its own day of the catalogue
(steps [480 r, 480 (r + 1)) of an N-day span) with no data-path collective:
weak scaling.
"""

from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2_20k_1d"
INTERVAL = 3.0 / 1440.0
THRESH = 5.0
METRIC = "object-days/s screened on 1 B200, mixed vs FP64 form, identical conj set"
UNIT = "object-days/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-chunks", type=int, default=10, help="time chunks of the overlapped polyjectory upload")
    ap.add_argument("--e2e-batch", type=int, default=48, help="conjunction steps per batch in the e2e call")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="screen only the first K conjunction steps (small cases for ncu captures)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the default launch shapes (shorter launch lists for profiling)")
    ap.add_argument("--configs", default="c1_1k_1d,c3_20k_shells_1d,c4_30k_7d,c5_60k_shells_3d",
                    help="other workloads timed after the headline one (comma-separated, '' for none)")
    ap.add_argument("--no-sgp4", action="store_true", help="skip the SGP4 polyjectory production timing")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """SM clock and throttle-reason samples taken during the timed region.

    Reads NVML every 5 ms (read-only queries) on a background thread, so that
    a timed region of a few hundred milliseconds still yields dozens of
    samples; falls back to ``nvidia-smi -lms 200`` when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
                   ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self.stop_ev = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _sample(self):
        nv, h = self.nvml
        try:
            if self.smax is None:
                self.smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), self.smax,
                                 nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
        except Exception as e:  # a failed query skips one sample
            self.errors.append(repr(e))

    def _poll(self):
        while not self.stop_ev.is_set():
            self._sample()
            time.sleep(0.005)

    def start(self):
        self.smax = None
        self.errors = []
        try:
            self.nvml = self._nvml_handle()
            self._sample()  # one sample at the start, whatever the thread does
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_ev.set()
            self.t.join(timeout=5)
            self._sample()  # and one at the end
            sm = [s[0] for s in self.samples]
            reasons = sorted({nm for _, _, bits in self.samples for nm, b in self.REASON_BITS if bits & b})
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": self.samples[0][1] if self.samples else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 5 ms",
                    "query_errors": len(self.errors)}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def state_meval_rate(pj, n_steps, calls=3):
    """State evaluation throughput through the public call (host arrays in
    and out): every object at the end time of each conjunction step.  The
    polyjectory is already on the device; the copies of the times in and of
    the states out (56 B per evaluation) are inside the timed region."""
    tm = np.minimum((np.arange(n_steps) + 1) * INTERVAL, pj.maxT) - 1e-9
    out = np.empty((pj.n_objs, n_steps, 7))
    pj.state_meval(time=tm, out=out)  # warm-up (uploads the polyjectory once)
    t0 = time.perf_counter()
    for _ in range(calls):
        pj.state_meval(time=tm, out=out)
    dt = (time.perf_counter() - t0) / calls
    n = pj.n_objs * n_steps
    return {"evals_per_s": n / dt, "ms_per_call": dt * 1e3, "evals_per_call": n,
            "d2h_bytes_per_call": int(out.nbytes), "valid_fraction": float(np.mean(~np.isnan(out[:, :, 0]))),
            "timing": "host wall clock around the blocking call, mean of 3 after 1 warm-up"}


def step_items(pj, s0, s1):
    """Number of (object, segment) pairs overlapping each step in [s0, s1):
    the AABB stage's work units."""
    a = pj.arrays
    ends = np.minimum((np.arange(s0, s1) + 1) * INTERVAL, a["maxT"])
    begins = np.arange(s0, s1) * INTERVAL
    total = 0
    for i in range(a["n_objs"]):
        ns = int(a["traj_offsets"][i, 1])
        if ns == 0:
            continue
        off = int(a["time_offsets"][i])
        t = a["time"][off:off + ns + 1]
        # segments [t[k], t[k+1]) overlapping [b, e): t[k] < e and t[k+1] > b
        lo = np.searchsorted(t[1:], begins, side="right")
        hi = np.searchsorted(t[:-1], ends, side="left")
        total += int(np.maximum(hi - lo, 0).sum())
    return total


def sample_blocks(n_steps, block, n_blocks):
    """Starts of n_blocks blocks of `block` consecutive conjunction steps
    spread evenly over [0, n_steps), in an order that alternates between the
    two halves of the span so that any prefix of the list is spread too."""
    n_blocks = max(1, min(n_blocks, n_steps // max(block, 1)))
    starts = [int(round(k * (n_steps - block) / max(n_blocks - 1, 1))) for k in range(n_blocks)]
    order = sorted(range(n_blocks), key=lambda k: (bin(k)[:1:-1] + "0" * 16)[:16])  # bit-reversed
    return [starts[k] for k in order]


def cpu_baseline(pj, seconds, n_threads, thresh=THRESH, n_steps=480):
    """The oracle port timed on a bounded sample: blocks of max(16, threads)
    consecutive conjunction steps (the oracle runs the steps of one call in
    parallel, one step per thread), the blocks spread over the whole span,
    until about `seconds` of wall time."""
    import oracle

    n = pj.n_objs
    block = max(16, n_threads)
    done, t_tot = 0, 0.0
    for s0 in sample_blocks(n_steps, block, n_steps // block):
        if t_tot >= seconds:
            break
        t0 = time.perf_counter()
        oracle.run(pj, thresh, INTERVAL, step_begin=s0, step_end=s0 + block, n_threads=n_threads)
        t_tot += time.perf_counter() - t0
        done += block
    value = n * done * INTERVAL / t_tot
    return {"value": value, "unit": UNIT, "cores": n_threads, "kind": "port",
            "sample": f"{done} of {n_steps} conjunction steps of the {n}-object span in blocks of {block} "
                      f"consecutive steps spread over the span, {t_tot:.1f} s wall"}


def workload_config(pj, conj_steps=480):
    """The bench line's `config` (both arms)."""
    a = pj.arrays
    return {"workload": f"{pj.n_objs} objects x 1 day per GPU, 3 min steps (480), 5 km threshold, "
                        "mixed form (FP64 narrow phase, FP32 broad phase on boxes that contain the "
                        "plain form's); the plain FP64 form is timed alongside",
            "objects": pj.n_objs, "days_per_gpu": 1, "conj_steps": conj_steps, "order": pj.poly_order,
            "polyjectory_gb": a["traj"].nbytes / 1e9,
            "l2": "inputs larger than L2 (polyjectory > 126 MB); no flush"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from mizuba_b200 import synth

    pj = synth.workload(args.workload)
    nt = os.cpu_count() or 1
    # The oracle runs the steps of one call in parallel (one step per
    # thread): each bench step is a block of max(16, threads) consecutive
    # conjunction steps, the blocks spread over the day.
    sample_steps = max(16, nt)
    import oracle

    starts = sample_blocks(480, sample_steps, max(args.steps, 1))
    for _ in range(args.warmup):
        oracle.run(pj, THRESH, INTERVAL, step_begin=starts[0], step_end=starts[0] + sample_steps, n_threads=nt)
    ts = []
    for k in range(args.steps):
        s0 = starts[k % len(starts)]
        t0 = time.perf_counter()
        oracle.run(pj, THRESH, INTERVAL, step_begin=s0, step_end=s0 + sample_steps, n_threads=nt)
        ts.append(time.perf_counter() - t0)
    t = max(statistics.mean(ts), 1e-9)
    value = pj.n_objs * sample_steps * INTERVAL / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(pj),
        "reference_sample": f"the reference algorithm (plain FP64) on {sample_steps} consecutive conjunction "
                            "steps per bench step, blocks spread over the day",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port",
                         "sample": f"{sample_steps} consecutive conjunction steps per bench step, "
                                   "blocks spread over the day"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "mizuba needs heyoka/TBB/Boost (absent): its CPU algorithm runs as the C++ restatement in oracle/",
    }
    print(json.dumps(line), flush=True)


def time_calls(fn, warmup, steps):
    """CUDA-event time of each of `steps` calls of fn() after warm-up calls;
    returns the median (ms), all of them, and the last result.  The median
    keeps a call that waited for the driver to map new pool memory from
    standing for the workload."""
    import torch

    for _ in range(warmup):
        r = fn()
        del r
    torch.cuda.synchronize()
    gc.collect()
    gc.disable()
    times, last = [], None
    for k in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
        if k == steps - 1:
            last = r
        else:
            del r
    gc.enable()
    return statistics.median(times), times, last


def config_line(name, tuning, n_threads, cpu_seconds):
    """One more workload at its full size: both forms device-resident (two
    warm-up calls, the median of three timed calls each), pair counts of both forms (the mixed
    form's superset ratio), and the oracle on a bounded sample of the same
    span on the host cores."""
    from mizuba_b200 import synth
    from mizuba_b200.conjunctions import device_conjunctions, to_device

    w = synth.WORKLOADS[name]
    t0 = time.perf_counter()
    pj = synth.workload(name)
    build_s = time.perf_counter() - t0
    dev = to_device(pj)
    S = int(math.ceil(pj.maxT / INTERVAL))
    out = {"objects": pj.n_objs, "days": w["days"], "conj_steps": S, "thresh_km": w["thresh"],
           "polyjectory_gb": pj.arrays["traj"].nbytes / 1e9, "host_build_s": build_s}
    if tuning is None:
        # Launch shapes tuned on this workload's own first batch (reported).
        from mizuba_b200.autotune import autotune

        tuning = autotune(dev, w["thresh"], INTERVAL, form="mixed")
        out["autotune"] = tuning
    res = {}
    for form in ("plain", "mixed"):
        ms, all_ms, r = time_calls(lambda: device_conjunctions(dev, w["thresh"], INTERVAL, form=form, tuning=tuning),
                                   2, 3)
        res[form] = r
        out[form] = {"ms_per_span": ms, "ms_per_call": all_ms, "object_days_per_s": pj.n_objs * w["days"] / (ms / 1e3),
                     "stage_ms": r.stage_ms, "pairs": int(r._L.mzb_result_n_bp(r._h)),
                     "conjunctions": int(r._L.mzb_result_n_conj(r._h))}
    cp, cm = res["plain"].conjunctions, res["mixed"].conjunctions
    same = len(cp) == len(cm) and bool(np.array_equal(np.sort(cp.view(np.uint8).reshape(len(cp), -1), axis=0),
                                                      np.sort(cm.view(np.uint8).reshape(len(cm), -1), axis=0)))
    out["mixed_over_plain"] = out["plain"]["ms_per_span"] / out["mixed"]["ms_per_span"]
    out["pair_superset_ratio"] = out["mixed"]["pairs"] / max(out["plain"]["pairs"], 1)
    out["same_conjunction_records"] = same
    del res, cp, cm
    out["cpu_baseline"] = cpu_baseline(pj, cpu_seconds, n_threads, thresh=w["thresh"], n_steps=S)
    del dev
    pj._device = None
    return out


def sgp4_line(n_threads, seconds):
    """SGP4 polyjectory production of the reference's 26,389-object
    catalogue (tests/golden/gpes.npz) over one day on the GPU, through the
    public call (element sets in, host arrays out); the oracle's serial
    restatement on the reference propagator times a sample beside it."""
    import torch

    from mizuba_b200 import make_sgp4_polyjectory

    g = np.load(os.path.join(ROOT, "tests", "golden", "gpes.npz"))["strack_20240705"]
    jd = 2460497.0
    make_sgp4_polyjectory(g[:500], jd, jd + 1.0)  # warm-up
    torch.cuda.synchronize()
    ts = []
    for _ in range(2):
        t0 = time.perf_counter()
        pj, _ = make_sgp4_polyjectory(g, jd, jd + 1.0)
        ts.append(time.perf_counter() - t0)
    st = pj.status
    n_ok = int(np.sum(st == 0))
    t = min(ts)
    segs = int(pj.arrays["traj_offsets"][:, 1].sum())
    out = {"element_sets": len(g), "objects": pj.n_objs, "objects_ok": n_ok, "segments": segs,
           "s_per_call": t, "object_days_per_s": n_ok / t,
           "timing": "host clock around the blocking call (element sets in, host arrays out), best of 2",
           "device_ms": pj.production_ms,
           "device_object_days_per_s": n_ok / (sum(pj.production_ms.values()) / 1e3),
           "output_gb": segs * 133 * 8 / 1e9}
    try:
        import oracle

        if oracle.sgp4_ref_lib() is not None:
            # One element set per object in this catalogue: object k is row k.
            near = g[st == 0] if len(st) == len(g) else g[:0]
            near = near[np.random.default_rng(0).permutation(len(near))]
            done, t_cpu, k = 0, 0.0, 0
            while t_cpu < seconds and k < len(near):
                part = near[k:k + 50]
                t0 = time.perf_counter()
                oracle.sgp4_polyjectory(part, jd, jd + 1.0)
                t_cpu += time.perf_counter() - t0
                done += len(part)
                k += 50
            out["cpu_baseline"] = {"value": done / t_cpu, "unit": "object-days/s", "cores": 1, "kind": "port",
                                   "sample": f"{done} element sets of the catalogue over 1 day, serial restatement "
                                             f"on the reference's SGP4 propagator, {t_cpu:.1f} s"}
    except Exception as e:  # the checker's absence must not fail the bench
        out["cpu_baseline"] = {"unavailable": repr(e)}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = dist_env()
    import torch

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import mizuba_b200
    from mizuba_b200 import _native, synth
    from mizuba_b200.conjunctions import device_conjunctions, to_device

    _native.core()  # fail loudly if the CUDA library is missing
    # Each rank screens day `rank` of the catalogue.
    pj = synth.workload(args.workload, t_start=float(rank))
    S_day = 480
    srange = (rank * S_day, (rank + 1) * S_day)
    if args.profile_steps:
        S_day = args.profile_steps
        srange = (rank * 480, rank * 480 + S_day)
    dev = to_device(pj)
    full = (srange == (0, 480))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    from mizuba_b200.shard import max_over_ranks

    # Launch shapes tuned once on this rank's own steps (not timed; reported).
    from mizuba_b200.autotune import autotune

    if args.no_autotune:
        tuning = {"bvh_threads": 0, "broad_walk": 0, "sort_threads": 512, "defaults": True}
    else:
        tuning = autotune(dev, THRESH, INTERVAL, form="mixed", step_range=srange)

    def one(form):
        return device_conjunctions(dev, THRESH, INTERVAL, step_range=None if full else srange, form=form,
                                   tuning=tuning)

    def timed(form, sampler=None):
        """W warm-up calls, then K timed calls (CUDA events, max over ranks)."""
        for _ in range(args.warmup):
            r = one(form)
            del r
        if sampler:
            sampler.start()
        # No cyclic garbage collection inside the timed region: a full pass
        # over the process's objects can stall the host for tens of ms.
        gc.collect()
        gc.disable()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launches, acc, last = 0, {}, None
        walls, per_call = [], []
        for k in range(args.steps):
            w0 = time.perf_counter()
            r = one(form)
            walls.append((time.perf_counter() - w0) * 1e3)
            per_call.append(round(r.stage_ms["total"], 3))
            launches += r.n_launches
            for key, v in r.stage_ms.items():
                acc[key] = acc.get(key, 0.0) + v
            if k == args.steps - 1:
                last = r
            else:
                del r
        e1.record()
        torch.cuda.synchronize()
        barrier()
        gc.enable()
        clocks = sampler.stop() if sampler else None
        t = max_over_ranks(e0.elapsed_time(e1) / args.steps, device="cuda")
        acc_avg = {k: v / args.steps for k, v in acc.items()}
        acc_avg["call_wall_ms"] = {"min": min(walls), "median": statistics.median(walls), "max": max(walls)}
        acc_avg["stage_total_ms_per_call"] = per_call
        return t, acc_avg, launches, last, clocks

    sampler = ClockSampler(local) if rank == 0 else None
    ms_plain, stage_plain, launches_plain, res_plain, _ = timed("plain")
    ms, stage_avg, launches, res_mixed, clocks = timed("mixed", sampler)
    np_rep = res_mixed.np_report
    np_split = res_mixed.narrow_split
    np_rep_plain = res_plain.np_report
    # The two forms must give the same conjunctions: identical (i, j)
    # multisets, matched TCA / DCA differences; pair counts of both.
    cp, cm = res_plain.conjunctions, res_mixed.conjunctions
    n_conj = int(len(cm))
    same_pairs = sorted(zip(cp["i"].tolist(), cp["j"].tolist())) == sorted(zip(cm["i"].tolist(), cm["j"].tolist()))
    ident = {"plain_conj": int(len(cp)), "mixed_conj": int(len(cm)), "same_ij_multiset": bool(same_pairs)}
    if same_pairs and len(cp):
        op = np.lexsort((cp["tca"], cp["j"], cp["i"]))
        om = np.lexsort((cm["tca"], cm["j"], cm["i"]))
        ident["max_abs_dtca_s"] = float(np.max(np.abs(cp["tca"][op] - cm["tca"][om])) * 86400.0)
        ident["max_rel_ddca"] = float(np.max(np.abs(cp["dca"][op] - cm["dca"][om])
                                             / np.maximum(cp["dca"][op], 1e-300)))
    ident["pairs_plain"] = int(res_plain._L.mzb_result_n_bp(res_plain._h))
    ident["pairs_mixed"] = int(res_mixed._L.mzb_result_n_bp(res_mixed._h))
    ident["pair_superset_ratio"] = ident["pairs_mixed"] / max(ident["pairs_plain"], 1)
    broad_visits = res_mixed.broad_visits
    res_mixed_tree_nodes = int(res_mixed._L.mzb_result_n_tree_nodes(res_mixed._h))
    del res_plain, res_mixed
    obj_days = pj.n_objs * S_day / 480.0
    value = obj_days * world / (ms / 1e3)
    value_plain = obj_days * world / (ms_plain / 1e3)

    # ---- end to end through the C ABI from pinned host memory
    a = pj.arrays
    pinned_in = {}
    for key in ("traj", "traj_offsets", "time", "time_offsets"):
        src = a[key]
        t = torch.empty(src.nbytes, dtype=torch.uint8, pin_memory=True)
        view = t.numpy().view(src.dtype).reshape(src.shape)
        view[...] = src
        pinned_in[key] = (t, view)
    h2d = sum(v[1].nbytes for v in pinned_in.values())
    import ctypes as ct

    L = _native.core()

    outs = {}

    def pinned(key, nbytes):
        buf = outs.get(key)
        if buf is None or buf[1].nbytes < nbytes:
            t = torch.empty(max(nbytes, 1), dtype=torch.uint8, pin_memory=True)
            buf = (t, t.numpy())
            outs[key] = buf
        return buf[1]

    # Overlapped upload: the polyjectory is packed by host threads and copied
    # up in E2E_CHUNKS time chunks while the screening runs in batches of
    # E2E_SPB steps (chunk and batch boundaries coincide on the 480-step day).
    E2E_CHUNKS, E2E_SPB = args.e2e_chunks, args.e2e_batch

    def e2e_once(overlap=True):
        """Host arrays in, host arrays out, through the C ABI: upload the
        polyjectory (by time chunk, overlapping the screening, unless
        overlap is False), screen with the per-step arrays and trees streamed
        into pinned host memory while the later stages compute
        (mzb_conjunctions_stream), then copy the pairs and conjunctions."""
        h = ct.c_void_p()
        p = pinned
        t0 = time.perf_counter()
        args_pj = (pinned_in["traj"][1].ctypes.data, a["traj"].size, pinned_in["traj_offsets"][1].ctypes.data,
                   pinned_in["time"][1].ctypes.data, a["time"].size, pinned_in["time_offsets"][1].ctypes.data,
                   a["n_objs"], a["order"], a["maxT"])
        if overlap:
            rc = L.mzb_pj_create_async(*args_pj, E2E_CHUNKS, ct.byref(h))
        else:
            rc = L.mzb_pj_create(*args_pj, ct.byref(h))
        assert rc == 0, L.mzb_last_error()
        S, N = srange[1] - srange[0], a["n_objs"]
        opts = _native.MzbOpts()
        opts.form = 1
        if overlap:
            opts.steps_per_batch = E2E_SPB
        opts.bvh_threads = int(tuning["bvh_threads"])
        opts.broad_walk = int(tuning["broad_walk"])
        opts.sort_threads = int(tuning["sort_threads"])
        if not full:
            opts.step_begin, opts.step_end = srange
        dst = _native.MzbHostOutputs()
        dense = (("aabbs", S * (N + 1) * 32), ("srt_aabbs", S * (N + 1) * 32), ("mcodes", S * N * 8),
                 ("srt_mcodes", S * N * 8), ("srt_idx", S * N * 4), ("cd_end_times", S * 8))
        for key, nb in dense:
            setattr(dst, key, p(key, nb).ctypes.data)
        dst.trees_cap = S * (2 * N - 1)
        dst.trees = p("trees", dst.trees_cap * 48).ctypes.data
        rh = ct.c_void_p()
        t1 = time.perf_counter()
        rc = L.mzb_conjunctions_stream(h, THRESH, INTERVAL, None, ct.byref(opts), ct.byref(dst), ct.byref(rh))
        assert rc == 0, L.mzb_last_error()
        t2 = time.perf_counter()
        nbytes = sum(nb for _, nb in dense) + int(L.mzb_result_n_tree_nodes(rh)) * 48
        nb = S * 16
        assert L.mzb_result_tree_offsets(rh, p("toff", nb).ctypes.data) == 0
        assert L.mzb_result_bp_offsets(rh, p("bpoff", nb).ctypes.data) == 0
        nbytes += 2 * nb
        nb = int(L.mzb_result_n_bp(rh)) * 8
        assert L.mzb_result_copy_bp(rh, p("bp", nb).ctypes.data) == 0
        nbytes += nb
        nb = int(L.mzb_result_n_conj(rh)) * 120
        assert L.mzb_result_copy_conj(rh, p("conj", nb).ctypes.data) == 0
        nbytes += nb
        t3 = time.perf_counter()
        L.mzb_result_free(rh)
        L.mzb_pj_free(h)
        e2e_split.append((t1 - t0, t2 - t1, t3 - t2))
        return nbytes

    e2e_split = []
    e2e_ms, e2e_sync_ms, d2h = float("nan"), float("nan"), 0
    if not args.no_e2e:
        d2h = e2e_once()  # warm-up (also sizes the D2H volume)
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.e2e_steps):
            e2e_once()
        e1.record()
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1) / args.e2e_steps
        # The same call with the upload finished before the screening starts
        # (mzb_pj_create, one batch), for comparison: one warm-up call (its
        # batch shape differs, so the scratch cache may grow), one timed.
        e2e_once(overlap=False)
        e2e_split.pop()
        e0.record()
        e2e_once(overlap=False)
        e1.record()
        torch.cuda.synchronize()
        e2e_sync_ms = e0.elapsed_time(e1)
        e2e_split.pop()
    e2e_ms = max_over_ranks(e2e_ms, device="cuda")
    e2e_value = obj_days * world / (e2e_ms / 1e3)

    # ---- roofline of the dominant stage
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    traffic = {}
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            traffic = json.load(f)
    except (OSError, ValueError):
        pass
    def traffic_of(*kernels):
        """DRAM bytes of the named kernels per full-day launch (None if any
        was not captured)."""
        vals = [traffic.get(k) for k in kernels]
        return None if any(v is None for v in vals) else int(sum(vals))

    n = pj.poly_order
    m = n + 1
    roof = None
    if rank == 0:
        rate = ct.c_double(0.0)
        assert L.mzb_measure_fp64_rate(ct.byref(rate)) == 0, L.mzb_last_error()
        fp64_peak = rate.value / 1e12  # DFMA instructions/s -> TOP/s (one op per FP64 instruction)
        # Narrow phase, per item (one pair of overlapping segments).  Plain
        # form: the reference's formulation (translation of 3 + 3
        # coordinates, Horner at m nodes for 6 polynomials, dist^2,
        # Bjorck-Pereyra, Cargo-Shisha).  Mixed form: FMA Horner of 6
        # polynomials at m shifted nodes, dist^2, Bjorck-Pereyra with
        # reciprocals, Cargo-Shisha on [0, 1].
        ops_plain = (2 * 3 * (3 * m * (m + 1) // 2 + n) + 2 * 6 * m * n + 8 * m
                     + (3 * n * (n + 1) // 2 + n * (n + 1)) + (3 * n + m + n * (n + 1) // 2 + 2 * m))
        ops_mixed = 6 * m * n + 3 * m + 3 * m + 3 * n * (n + 1) // 2 + m + n * (n + 1) // 2 + 2 * n
        # Mixed narrow stage: the distance screen on every item (about 65
        # FP64 operations from the two stored linear models), the FMA
        # prefilter on the items that pass it, the reference formulation on
        # the prefilter's survivors.
        ops_screen = 65
        mixed_narrow_ops = np_rep[0] * ops_screen + np_split[0] * ops_mixed + np_split[1] * ops_plain

        def fp64_roof(stage, kernel, units, ops, t_ms, extra=None, kernels=None):
            ach = units * ops / (t_ms / 1e3) / 1e12
            r = {"stage": stage, "kernel": kernel, "bound": "fp64", "achieved": ach, "peak": fp64_peak,
                 "unit": "TOP/s", "frac": ach / fp64_peak, "traffic": traffic_of(*(kernels or [kernel])),
                 "units_per_launch": units, "algorithmic_ops_per_unit": ops,
                 "peak_source": "measured DFMA issue rate (mzb_measure_fp64_rate), one op per FP64 instruction"}
            r.update(extra or {})
            return r

        n_seg_items = step_items(pj, srange[0], srange[1])
        ops_seg_plain = 4 * (m * (m + 1) + (m * (m + 1) // 2 - m) + 2 * (n - 1) + 2 * m + n * (n + 1) // 2 + 2)
        # Mixed enclosure per variable, plus the screen model of x, y, z
        # (value and derivative by Horner, the curvature bound: 3 n each).
        ops_seg_mixed = 4 * (n + n * (n + 1) // 2 + 3 * m + n * (n + 1) // 2 + 2 * n + 4) + 3 * 3 * n
        seg_bytes = {"algorithmic_bytes_per_unit": 4 * m * 8 + 16}
        stages = {
            "narrow": fp64_roof("narrow", "k_items_screen + k_narrow_mixed + k_narrow", np_rep[0],
                                mixed_narrow_ops / max(np_rep[0], 1), stage_avg["narrow"],
                                {"items_screened": np_rep[0], "items_prefiltered": np_split[0],
                                 "items_exact": np_split[1],
                                 "ops_per_item": {"screen": ops_screen, "prefilter": ops_mixed,
                                                  "exact": ops_plain}},
                                kernels=["k_items_screen", "k_narrow_mixed", "k_narrow_survivors"]),
            "aabb": fp64_roof("aabb", "k_aabb_mixed", n_seg_items, ops_seg_mixed, stage_avg["aabb"], seg_bytes,
                              kernels=["k_aabb_mixed", "k_aabb_mixed_more"]),
            "narrow_plain_form": fp64_roof("narrow", "k_narrow", np_rep_plain[0], ops_plain, stage_plain["narrow"]),
            "aabb_plain_form": fp64_roof("aabb", "k_aabb", n_seg_items, ops_seg_plain, stage_plain["aabb"],
                                         seg_bytes),
        }
        # BVH: the trees written (48 B per node) and the sorted codes and
        # boxes read (40 B per object and step).  Broad phase: one 32-byte
        # walk node per visit (device counter) and 8 B per pair written.
        tree_nodes = int(res_mixed_tree_nodes)
        bvh_bytes = tree_nodes * 48 + pj.n_objs * S_day * 40
        bvh_ach = bvh_bytes / (stage_avg["bvh"] / 1e3) / 1e9
        stages["bvh"] = {"stage": "bvh", "kernel": "k_bvh_flat + k_walk_nodes", "bound": "hbm", "achieved": bvh_ach,
                         "peak": hbm_peak, "unit": "GB/s", "frac": bvh_ach / hbm_peak,
                         "traffic": traffic_of("k_bvh_flat", "k_walk_nodes"), "tree_nodes": tree_nodes,
                         "algorithmic_bytes": bvh_bytes, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
        broad_bytes = broad_visits * 32 + ident["pairs_mixed"] * 8
        broad_ach = broad_bytes / (stage_avg["broad"] / 1e3) / 1e9
        stages["broad"] = {"stage": "broad", "kernel": "k_broad_half + scan + copy", "bound": "hbm",
                           "achieved": broad_ach, "peak": hbm_peak, "unit": "GB/s", "frac": broad_ach / hbm_peak,
                           "traffic": traffic_of("k_broad_half"), "node_visits": broad_visits,
                           "node_visits_per_s": broad_visits / (stage_avg["broad"] / 1e3),
                           "visits_per_walk": broad_visits / max(pj.n_objs * S_day, 1),
                           "algorithmic_bytes": broad_bytes, "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
        # Morton + sort + gather: 148 B per object and step (HBM roofline).
        ms_ach = 148 * pj.n_objs * S_day / (stage_avg["morton_sort"] / 1e3) / 1e9
        stages["morton_sort"] = {"stage": "morton_sort", "kernel": "k_morton + k_sort_step", "bound": "hbm",
                                 "achieved": ms_ach, "peak": hbm_peak, "unit": "GB/s", "frac": ms_ach / hbm_peak,
                                 "traffic": traffic_of("k_sort_step"),
                                 "peak_source": "MEASURED_PEAKS.json hbm_gbs"}
        dominant = max(("narrow", "aabb", "bvh", "broad", "morton_sort"), key=lambda k: stage_avg.get(k, 0.0))
        roof = dict(stages[dominant])
        roof["stages"] = stages
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(pj, S_day),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "ms_per_step": e2e_ms,
                # Average link rates over the call (both directions overlap).
                "h2d_gbs": h2d / (e2e_ms / 1e3) / 1e9 if e2e_ms == e2e_ms and e2e_ms > 0 else None,
                "d2h_gbs": d2h / (e2e_ms / 1e3) / 1e9 if e2e_ms == e2e_ms and e2e_ms > 0 else None,
                "split_ms": None if not e2e_split else {
                    "create_async": 1e3 * statistics.median(x[0] for x in e2e_split[1:] or e2e_split),
                    "upload_screen_and_stream": 1e3 * statistics.median(x[1] for x in e2e_split[1:] or e2e_split),
                    "pairs_and_conj_copies": 1e3 * statistics.median(x[2] for x in e2e_split[1:] or e2e_split),
                    "timing": "host clock around each blocking call, median of the timed calls"},
                "upload": f"mzb_pj_create_async, {E2E_CHUNKS} time chunks packed by host threads into pinned "
                          f"pieces and copied up while batches of {E2E_SPB} steps screen",
                "sync_upload": {"value": obj_days * world / (e2e_sync_ms / 1e3) if e2e_sync_ms == e2e_sync_ms
                                else None, "ms_per_step": e2e_sync_ms,
                                "note": "mzb_pj_create (upload finished first), one batch; one call after one warm-up"}},
        "gpu_launches": int(launches),
        "stage_ms": stage_avg,
        "np_report": np_rep,
        "n_conj": n_conj,
        "fp64_form": {"value": value_plain, "ms_per_step": ms_plain, "stage_ms": stage_plain,
                      "np_report": np_rep_plain, "gpu_launches": int(launches_plain)},
        "mixed_over_fp64": value / value_plain,
        "forms_identity": ident,
        "roofline": roof,
        "clocks": clocks,
        "autotune": tuning,
    }
    if rank == 0 and world == 1 and not args.no_e2e:
        line["state_meval"] = state_meval_rate(pj, S_day)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(pj, args.cpu_seconds, os.cpu_count() or 1)
    if rank == 0 and world == 1 and args.configs and not args.profile_steps:
        # The other workloads at their full sizes (extra keys; the headline
        # stays the 20,000-object day).
        del dev
        pj._device = None
        line["configs"] = {}
        for name in [c for c in args.configs.split(",") if c]:
            line["configs"][name] = config_line(name, None if not args.no_autotune else tuning,
                                                os.cpu_count() or 1, 4.0)
    if rank == 0 and world == 1 and not args.no_sgp4 and not args.profile_steps:
        line["sgp4_production"] = sgp4_line(os.cpu_count() or 1, 5.0)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
