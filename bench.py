#!/usr/bin/env python
"""PU200-shaped events/s of the LST object-building chain on B200.

A step is one batch of seeded PU200-shaped events (generator configuration 2:
~20 hard tracks + Poisson(200) vertices x Poisson(60) particles, 1% noise
hits) taken through every stage: hit preparation, mini-doublets, segments,
triplets, quintuplets (reference-weight DNN), pLS cleaning, pT5, pT3 and
track candidates.

Reported:
  value        batched throughput: the whole batch in one launch per kernel,
               replayed from a CUDA graph, inputs already resident on the
               device (lst_batch_ingest + lst_batch_run_graph), events/s over
               all ranks
  drop_in      the same events one at a time (per-event launches), events/s
  e2e          batched through the C ABI from pinned host buffers: packed
               input upload, all stages, LST::getOutput-style track-candidate
               hit lists copied back (lst_batch_upload + lst_batch_run +
               lst_batch_get_output), events/s; e2e_drop_in is the per-event
               C ABI (add_hits + add_pixel_segments from host arrays, stages,
               get_output) event by event
  roofline     the kernel with the largest share of device time, its
               algorithmic bytes per launch over its CUDA-event duration
  cpu_baseline the reference CPU backend (oracle/_ref, reference compiler
               flags) on the host cores, one event per thread
  t5_classifier  T5 efficiency and fake rate (truth-matched quintuplet
               candidates at the classifier decision) and batched events/s for
               the reference-weight DNN, the retrained DNN and cut-only

--impl reference times only the reference CPU backend on this workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "PU200 events/s on 1 B200 (batched 64/launch; per-event drop-in reported beside it)"
HBM_FALLBACK_GBS = 6650.0

# Algorithmic bytes per object of the dominant kernels: each input read once,
# each output record written once, in the reference's field widths.
#   MD: 40 B per hit in (x, y, z, rt, phi, eta, 4 edges) + 134 B per MD out
#   LS: 44 B per MD in + 80 B per module (module map) + 44 B per LS out
#   T3: 24 B per LS + 20 B per MD in + 60 B per T3 out
#   T5 (kT5Eval): 60 B per T3 + 56 B per MD in + 110 B per T5 out
#   pT3/pT5 (kPixEval): 76 B per pLS + 4 B per connected-module entry + 60 B per
#            T3 (or 110 B per T5) in + 100 B per pT3/pT5 out
ALGO_BYTES = {
    "kCreateMD": lambda c: 40 * c["nHits"] + 134 * c["nMD"],
    "kCreateLS": lambda c: 44 * c["nMD"] + 80 * c["nLower"] + 44 * c["nLS"],
    "kCreateT3": lambda c: 24 * c["nLS"] + 20 * c["nMD"] + 60 * c["nT3"],
    "kT5Eval": lambda c: 60 * c["nT3"] + 56 * c["nMD"] + 110 * c["nT5"],
    "kPixEval<3>": lambda c: 76 * c["nPLS"] + 4 * 40 * c["nPLS"] + 60 * c["nT3"] + 100 * c["nPT3"],
    "kPixEval<5>": lambda c: 76 * c["nPLS"] + 4 * 40 * c["nPLS"] + 110 * c["nT5"] + 100 * c["nPT5"],
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def rank_first_event(rank: int, batch: int) -> int:
    """First generator index of a rank's batch: ranks take disjoint events."""
    return rank * batch


def reduce_max(value: float, world: int, device=None) -> float:
    """Max of `value` over the ranks (the timing rule for N > 1)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as tdist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def generate(config: int, first: int, n: int, workers: int):
    from tracklooper_b200 import gen

    with ThreadPoolExecutor(max_workers=max(1, workers)) as pool:
        return list(pool.map(lambda i: gen.generate_event(config, first + i), range(n)))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi takes a moment to start: begin the timed region at its first sample
        t0 = time.time()
        while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
            time.sleep(0.005)
        self.lines.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


def committed_issue_slots(kernel: str):
    """(IPC, fraction of the 4 issue slots per SM, how it was captured) of
    `kernel` from the committed ncu summary (profiles/issue_slots.txt), or
    (None, None, None)."""
    path = os.path.join(ROOT, "profiles", "issue_slots.txt")
    note = []
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("#"):
                    note.append(line[1:].strip())
                    continue
                parts = line.split()
                if len(parts) >= 3 and parts[0] == kernel:
                    return float(parts[1]), float(parts[2]), " ".join(note)
    except OSError:
        pass
    return None, None, None


def committed_traffic(kernel: str):
    """(DRAM bytes per launch of `kernel`, how they were captured) from the
    committed ncu summary (profiles/dram_traffic.txt: '# ' comment lines
    saying how the capture was made, then '<kernel> <bytes>' lines);
    (None, None) if no capture of that kernel is committed."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    note = []
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("#"):
                    note.append(line[1:].strip())
                    continue
                parts = line.split()
                if len(parts) >= 2 and parts[0] == kernel:
                    return float(parts[1]), " ".join(note)
    except OSError:
        pass
    return None, None


# --------------------------------------------------------------------- ours
def run_ours(args, rank, world, local, events):
    import torch
    import torch.distributed as tdist

    from tracklooper_b200 import lst

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    B = len(events)
    es = lst.ES(device=local)
    max_hits = max(e.n_hits for e in events)
    max_hits = ((max_hits + 4095) // 4096) * 4096
    eset = lst.EventSet(es, n_slots=B, max_hits=max_hits)
    stream = torch.cuda.ExternalStream(eset.stream(), device=dev)

    blob_np, offsets = lst.pack_events(events)
    pinned = torch.empty(blob_np.nbytes, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = blob_np
    blob = pinned.numpy()
    in_bytes = int(blob.nbytes)

    # output buffers (pinned)
    tc_cap = 31000 * B
    out_hits = torch.empty(tc_cap * 14, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    out_len = torch.empty(tc_cap, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    out_seed = torch.empty(tc_cap, dtype=torch.int32, pin_memory=True).numpy()
    out_type = torch.empty(tc_cap, dtype=torch.int16, pin_memory=True).numpy()
    tco = np.zeros(B + 1, np.uint64)
    hco = np.zeros(B + 1, np.uint64)
    outs = lst.Output(out_hits.ctypes.data, out_hits.size, out_len.ctypes.data, out_seed.ctypes.data,
                      out_type.ctypes.data, out_len.size, tco.ctypes.data, hco.ctypes.data)
    lib = lst.library()
    import ctypes

    def get_output():
        lst._check(lib.lst_batch_get_output(eset.handle, 0, B, ctypes.byref(outs)), "lst_batch_get_output")
        n_tc, n_h = int(tco[-1]), int(hco[-1])
        return n_tc * (4 + 4 + 2) + n_h * 4 + 2 * (B + 1) * 8

    # first pass: upload + all stages + output (also a correctness gate on status bits)
    eset.upload_packed(0, blob, offsets)
    eset.run(0, B)
    counts = eset.batch_counts(0, B)
    bad = [i for i, c in enumerate(counts) if c["status"] & ~0x30]
    if bad:
        raise RuntimeError(f"events with input errors: {bad[:5]}")
    d2h_bytes = get_output()
    n_tc0, n_h0 = int(tco[-1]), int(hco[-1])
    batched_out = [a.copy() for a in (out_hits[:n_h0], out_len[:n_tc0], out_seed[:n_tc0], out_type[:n_tc0], tco, hco)]

    # launch shapes: the cached autotuner entry for this geometry, device,
    # batch size and build, or a fresh sweep on these (resident) events
    tune_cache = os.environ.get("LST_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "tracklooper_b200", "autotune.txt")
    os.makedirs(os.path.dirname(tune_cache), exist_ok=True)
    t_tune = time.perf_counter()
    tuned_from = "cache" if eset.autotune_load(B, tune_cache) else "sweep"
    if tuned_from == "sweep":
        eset.autotune(0, B, tune_cache)
    tune_info = {"source": tuned_from, "seconds": round(time.perf_counter() - t_tune, 2),
                 "shapes": {k: list(v) for k, v in eset.launch_shapes().items()},
                 "geometry_hash": f"{es.geometry_hash():016x}"}
    eset.upload_packed(0, blob, offsets)
    # more event sets with the same resident inputs and launch shapes: the
    # batched steps go to the sets in turn, so that one batch's kernels fill
    # the SMs that another batch's kernel tails and small stages leave idle
    # (args.sets batches in flight, each set on its own stream)
    sets = [eset]
    for _ in range(args.sets - 1):
        e_ = lst.EventSet(es, n_slots=B, max_hits=max_hits)
        if not e_.autotune_load(B, tune_cache):
            raise RuntimeError("an added event set could not load the launch shapes of the first")
        e_.upload_packed(0, blob, offsets)
        sets.append(e_)
    streams = [torch.cuda.ExternalStream(e_.stream(), device=dev) for e_ in sets]
    turn = [0]

    def batched_step():
        eset.ingest(0, B)
        eset.run_graph(0, B)

    def pipelined_step():
        s_ = sets[turn[0] % len(sets)]
        turn[0] += 1
        s_.ingest(0, B)
        s_.run_graph(0, B)

    def dropin_step():
        # one event per launch sequence: each event's stages replayed as that
        # event's own CUDA graph
        for i in range(B):
            eset.ingest(i, 1)
            eset.run_graph(i, 1)

    def timed(step, k, sampler=None):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if world > 1:
            tdist.barrier()
        torch.cuda.synchronize()
        if sampler:
            sampler.start()
        l0 = sum(e_.launches() for e_ in sets)
        start.record(stream)
        for st_ in streams[1:]:
            st_.wait_stream(stream)  # the other sets' work starts after the start mark
        for _ in range(k):
            step()
        for st_ in streams[1:]:
            stream.wait_stream(st_)  # and the stop mark comes after every set's work
        stop.record(stream)
        stop.synchronize()
        l1 = sum(e_.launches() for e_ in sets)
        clocks = sampler.stop() if sampler else None
        torch.cuda.synchronize()
        ms = reduce_max(start.elapsed_time(stop), world, dev)
        return ms, l1 - l0, clocks

    # warm-up
    for _ in range(args.warmup):
        batched_step()
        pipelined_step()
    for _ in range(max(1, args.warmup // 2)):
        dropin_step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    ms_b, launches_b, clocks = timed(pipelined_step, args.steps, sampler)
    ms_b1, _, _ = timed(batched_step, args.steps)  # one set: the steps one after the other
    ms_d, _, _ = timed(dropin_step, max(1, args.steps // 2))
    steps_d = max(1, args.steps // 2)
    # the slots now hold the per-event (drop-in) results: the same lists?
    get_output()
    n_tc1, n_h1 = int(tco[-1]), int(hco[-1])
    dropin_out = (out_hits[:n_h1], out_len[:n_tc1], out_seed[:n_tc1], out_type[:n_tc1], tco, hco)
    same_lists = all(np.array_equal(a, b) for a, b in zip(batched_out, dropin_out))

    # e2e batched: host packed inputs -> device -> stages -> track-candidate
    # output on host.  Every step copies its inputs in and its outputs back.
    # Two event sets take the steps in turn, as a serving loop would: a step's
    # input copy (lst_batch_stage, on its set's copy stream) and the reading of
    # the previous step's output (lst_batch_get_output, on the other set's
    # stream) overlap the stages running on the GPU.
    def get_output_of(s):
        lst._check(lib.lst_batch_get_output(s.handle, 0, B, ctypes.byref(outs)), "lst_batch_get_output")

    def e2e_run(k):
        sets[0].stage(0, blob, offsets)
        prev = None
        for i in range(k):
            cur = sets[i % len(sets)]
            cur.ingest_staged()
            cur.run_graph(0, B)
            if i + 1 < k:
                sets[(i + 1) % len(sets)].stage(0, blob, offsets)
            if prev is not None:
                get_output_of(prev)
            prev = cur
        get_output_of(prev)

    e2e_run(2)
    # three timed repetitions, the median reported: the host side of the
    # copies and of lst_batch_get_output is exposed to host jitter
    ms_e_runs = [timed(lambda: e2e_run(args.steps), 1)[0] for _ in range(3)]
    ms_e = sorted(ms_e_runs)[1]
    mem_bytes = eset.memory_bytes()
    # the host -> device copy of one step's packed inputs alone, for the e2e
    # bound (the copies of consecutive steps cannot overlap one another)
    dev_in = torch.empty(in_bytes, dtype=torch.uint8, device=dev)
    h2d_ms = []
    for _ in range(4):
        a_ = torch.cuda.Event(enable_timing=True)
        b_ = torch.cuda.Event(enable_timing=True)
        a_.record()
        dev_in.copy_(pinned, non_blocking=True)
        b_.record()
        b_.synchronize()
        h2d_ms.append(a_.elapsed_time(b_))
    del dev_in
    h2d_gbs = in_bytes / (min(h2d_ms[1:]) * 1e-3) / 1e9

    # e2e drop-in: per-event C ABI calls with host arrays, event by event
    ev1 = lst.Event(es, event_set=eset, slot=0)

    def e2e_dropin_step():
        for i, inp in enumerate(events):
            e = lst.Event(es, event_set=eset, slot=i)
            e.run(inp)
            eset.output(i, 1)

    e2e_dropin_step()
    n_dropin_e2e = max(1, args.steps // 4)
    ms_de, _, _ = timed(e2e_dropin_step, n_dropin_e2e)
    del ev1

    # per-kernel device time (instrumented pass over the same batched steps,
    # launched directly because graph replays cannot be timed per kernel)
    eset.set_profiling(True)
    for _ in range(args.steps):
        eset.ingest(0, B)
        eset.run(0, B)
    prof = eset.profile()
    eset.set_profiling(False)

    # T5 selection methods in the loop: candidate-level truth-matched
    # efficiency / fake rate at the classifier stage (the probe) and batched
    # events/s, for the reference-weight DNN, the retrained DNN and cut-only
    from tracklooper_b200 import t5dnn

    probe = t5dnn.collect_candidates(es, events, batch=B, eset=eset)
    w_new, wp_new = t5dnn.retrained_weights()
    lab = probe["label"]
    classifier = {"candidates": int(lab.size), "true": int(lab.sum()),
                  "reference_dnn": t5dnn.metrics(probe["score"] > np.float32(t5dnn.REFERENCE_WP), lab),
                  "retrained_dnn": t5dnn.metrics(t5dnn.scores(probe, w_new, local) > wp_new, lab),
                  "cut_only": t5dnn.metrics(probe["cut"] != 0, lab)}
    eset.upload_packed(0, blob, offsets)
    k_m = max(2, args.steps // 2)
    from tracklooper_b200 import performance

    def tc_level():
        # track-candidate efficiency / fake / duplicate rates of the slots'
        # current outputs (the reference's definitions, performance.py)
        eset.sync()
        return performance.combine([performance.from_store(lambda f, i=i: eset.field(i, f), events[i])
                                    for i in range(B)])

    ms_ref, _, _ = timed(batched_step, k_m)
    tc_ref = tc_level()
    es.set_t5dnn_weights(w_new)
    es.set_t5dnn_threshold(wp_new)
    batched_step()
    ms_new, _, _ = timed(batched_step, k_m)
    tc_new = tc_level()
    es.set_t5dnn_weights(t5dnn.reference_weights())
    es.set_t5dnn_threshold(t5dnn.REFERENCE_WP)
    eset.set_t5_method(lst.T5_CUTS)
    batched_step()
    ms_cut, _, _ = timed(batched_step, k_m)
    tc_cut = tc_level()
    eset.set_t5_method(lst.T5_DNN)
    for key, ms_, tc in (("reference_dnn", ms_ref, tc_ref), ("retrained_dnn", ms_new, tc_new),
                         ("cut_only", ms_cut, tc_cut)):
        classifier[key]["events_per_s"] = B * world * k_m / (ms_ * 1e-3)
        classifier[key]["track_candidates"] = {
            "fake_rate": tc["fake_rate"], "duplicate_rate": tc["duplicate_rate"],
            "efficiency_hard": tc["hard"]["efficiency"], "efficiency_pileup": tc["pileup"]["efficiency"],
            "t5_tc": tc["by_type"]["T5"]["tc"], "t5_tc_fake_rate": tc["by_type"]["T5"]["fake_rate"]}
    classifier["retrained_working_point"] = wp_new
    classifier["level"] = ("quintuplet candidates reaching the classifier decision, this step's events; "
                           "track_candidates: the final track candidates (pT > 1 GeV, |eta| < 2.4 particles)")

    tot = sum(v[1] for v in prof.values())
    top = sorted(prof.items(), key=lambda kv: -kv[1][1])
    agg = {
        "nHits": sum(c["nHits"] for c in counts),
        "nMD": sum(c["nMiniDoublets"] for c in counts) + sum(2 * c["nPixelSegments"] for c in counts),
        "nLS": sum(c["nSegments"] for c in counts),
        "nT3": sum(c["nTriplets"] for c in counts),
        "nT5": sum(c["nQuintuplets"] for c in counts),
        "nPLS": sum(c["nPixelSegments"] for c in counts),
        "nPT3": sum(c["nPixelTriplets"] for c in counts),
        "nPT5": sum(c["nPixelQuintuplets"] for c in counts),
        "nTC": sum(c["nTrackCandidates"] for c in counts),
        "nLower": es.info["nLowerModules"] * B,
    }
    peak, peak_kind = hbm_peak()
    dominant = next((k for k, _ in top if k in ALGO_BYTES), top[0][0])
    dlaunches, dms = prof[dominant]
    algo = ALGO_BYTES[dominant](agg) if dominant in ALGO_BYTES else None
    achieved = (algo / (dms / dlaunches * 1e-3) / 1e9) if algo else None
    roofline = {
        "bound": "hbm",
        "kernel": dominant,
        "achieved": round(achieved, 2) if achieved else None,
        "peak": peak,
        "peak_kind": f"{peak_kind} (copy bandwidth)",
        "unit": "GB/s",
        "frac": round(achieved / peak, 5) if achieved else None,
        "traffic": committed_traffic(dominant)[0],
        "traffic_source": committed_traffic(dominant)[1],
        "algorithmic_bytes_per_launch": algo,
        "issue_slots": dict(zip(("ipc", "frac", "source"), committed_issue_slots(dominant))),
        "launch_ms": round(dms / dlaunches, 4),
        "share_of_device_time": round(dms / tot, 4) if tot else None,
    }
    kernel_table = {k: {"launches": v[0], "ms_per_step": round(v[1] / args.steps, 4),
                        "share": round(v[1] / tot, 4) if tot else None} for k, v in top[:12]}

    events_all = B * world
    value = events_all * args.steps / (ms_b * 1e-3)
    res = {
        "value": value,
        "ms_per_step": ms_b / args.steps,
        "one_set": {"value": events_all * args.steps / (ms_b1 * 1e-3), "unit": "events/s",
                    "ms_per_step": ms_b1 / args.steps,
                    "mode": "one event set, each step's stages after the previous step's"},
        "pipelining": f"{len(sets)} event sets with the same resident inputs take the steps in turn, each on its "
                      "own stream; ms_per_step is the timed region over the steps",
        "drop_in": {"value": events_all * steps_d / (ms_d * 1e-3), "unit": "events/s",
                    "ms_per_event": ms_d / steps_d / B,
                    "mode": "one event per launch sequence (lst_batch_ingest, then lst_batch_run_graph of that "
                            "event's slot: its stages as one CUDA graph)"},
        "batched_over_drop_in": (ms_d / steps_d) / (ms_b / args.steps),
        "batched_equals_drop_in": same_lists,
        "e2e": {"value": events_all * args.steps / (ms_e * 1e-3), "unit": "events/s",
                "runs": [round(events_all * args.steps / (t * 1e-3), 1) for t in ms_e_runs],
                "h2d_bytes_per_step": in_bytes + 8 * B, "d2h_bytes_per_step": d2h_bytes,
                "mode": f"batched C ABI from pinned host buffers, {len(sets)} event sets taking the steps in turn: each "
                        "step's packed inputs copied in (lst_batch_stage on its set's copy stream), "
                        "lst_batch_ingest_staged, lst_batch_run_graph, and its output read back "
                        "(lst_batch_get_output) while the next step's stages run",
                "h2d_gbs": round(h2d_gbs, 1),
                "h2d_bound_events_per_s": round(events_all / (in_bytes / (h2d_gbs * 1e9)), 1)},
        "e2e_drop_in": {"value": events_all * n_dropin_e2e / (ms_de * 1e-3), "unit": "events/s",
                        "mode": "per-event C ABI from host arrays (add_hits, add_pixel_segments, stages, output)"},
        "t5_classifier": classifier,
        "gpu_launches": launches_b,
        "clocks": clocks,
        "roofline": roofline,
        "kernels": kernel_table,
        # device time of all of a step's kernels (CUDA events around each,
        # direct launches) beside the graph-replayed step: the difference is
        # what the step's launch boundaries cost
        "kernels_sum_ms_per_step": round(tot / args.steps, 4),
        "launches_per_step": round(sum(v[0] for v in prof.values()) / args.steps, 1),
        "objects_per_event": {k: round(v / B, 1) for k, v in agg.items() if k != "nLower"},
        "device_memory_gb": round(len(sets) * mem_bytes / 1e9, 2),
        "autotune": tune_info,
        "l2": f"inputs larger than L2: {in_bytes / 1e6:.0f} MB of packed inputs per step plus the object arenas",
    }
    for e_ in sets[1:]:
        e_.close()
    eset.close()
    es.close()
    return res


# ----------------------------------------------------------- reference CPU
def run_reference_cpu(events, threads: int, min_events: int, budget_s: float = 0.0):
    """Reference CPU backend, one event per thread at a time, over at least
    min_events events and (when budget_s > 0) for at least budget_s seconds,
    cycling through the events; returns (events/s, events, threads, seconds)."""
    from oracle import reflib

    variant = "fast"
    if not reflib.available(variant):
        raise FileNotFoundError(reflib.library_path(variant))
    base = reflib.RefLST(variant)
    workers = [base] + [base.fork() for _ in range(threads - 1)]
    # warm one event per worker (page-in, allocator)
    n = max(min_events, threads)
    lock = threading.Lock()
    next_i = [0]
    done = [0]
    t_end = [None]

    def work(w):
        while True:
            with lock:
                i = next_i[0]
                if i >= n and time.perf_counter() - t0 >= budget_s:
                    return
                next_i[0] += 1
            w.run_event(events[i % len(events)])
            with lock:
                done[0] += 1

    t0 = time.perf_counter()
    ths = [threading.Thread(target=work, args=(w,)) for w in workers]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    dt = time.perf_counter() - t0
    for w in workers[1:]:
        w.close()
    base.close()
    return done[0] / dt, done[0], threads, dt


def reference_cpu_baseline(events, ncpu: int, min_events: int, budget_s: float = 12.0) -> dict:
    """The reference CPU backend on this host: all usable cores, then one
    thread, each a sustained sample of at least budget_s seconds (threads keep
    taking the next event until both the event count and the time are
    reached, so only the last wave of the whole sample has a tail)."""
    threads = cpu_threads(ncpu)
    r_all, n_all, th, dt_all = run_reference_cpu(events, threads, max(min_events, threads), budget_s=budget_s)
    r_one, n_one, _, dt_one = run_reference_cpu(events, 1, 1, budget_s=budget_s)
    return {"value": r_all, "unit": "events/s", "cores": th, "kind": "reference",
            "sample": f"{n_all} events of this batch (cycled), one event per thread on {th} threads, "
                      f"{dt_all:.1f} s wall, liblstref_fast.so (reference compiler flags)",
            "one_thread": {"value": r_one, "unit": "events/s", "cores": 1,
                           "sample": f"{n_one} events, {dt_one:.1f} s wall"},
            "host_cpus": ncpu}


def cpu_threads(ncpu: int) -> int:
    """Host threads for the reference CPU backend: all cores, bounded by memory
    (each in-flight reference event holds ~0.6 GB of object arenas)."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail_gb = int(line.split()[1]) / 1e6
                    return max(1, min(ncpu, int(avail_gb / 0.6)))
    except OSError:
        pass
    return ncpu


def launcher_command(argv, n_gpus: int, port: int) -> list:
    """The command that runs this script as n_gpus local ranks (one process
    per GPU), as the torchrun launch of a multi-GPU bench does."""
    return [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n_gpus}",
            "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)


def _free_port() -> int:
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--sets", type=int, default=2, choices=range(1, 5), metavar="{1..4}",
                    help="event sets taking the batched steps in turn")
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--cpu-events", type=int, default=0, help="reference CPU sample size (0: 2 per thread)")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    return args


def main(argv=None, runner=None, backend: str = "nccl"):
    """Runs the bench; `runner(args, rank, world, local, events)` replaces the
    GPU replica (run_ours) and `backend` the process-group backend, which is
    how the CPU tests drive the multi-rank harness with gloo."""
    argv = sys.argv[1:] if argv is None else list(argv)
    args = parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch as args.gpus local ranks
        rc = subprocess.call(launcher_command(argv, args.gpus, _free_port()))
        sys.exit(rc)
    rank, world, local = dist_env()
    if world != args.gpus and rank == 0:
        log(f"note: --gpus {args.gpus} but WORLD_SIZE={world}; running {world} ranks")
    ncpu = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)

    config = {"workload": f"PU200-shaped events (generator configuration {args.config}), batch of {args.batch} per GPU",
              "events_per_step_per_gpu": args.batch, "geometry": "OT800_IT615_pt0.8",
              "t5_selection": "reference-weight DNN", "parallelism": f"replicas x{world}",
              "event_sets_per_gpu": args.sets}
    base = {"metric": METRIC, "unit": "events/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator, PU200-shaped)", "config": config}

    if args.impl == "reference":
        if rank != 0:
            return
        events = generate(args.config, 0, args.batch, ncpu)
        threads = cpu_threads(ncpu)
        # warm-up: one event per thread (page-in, allocator)
        run_reference_cpu(events, threads, threads)
        # one sustained sample covering all steps' events (steps x batch), at
        # least 12 s, with threads taking the next event as they finish: no
        # per-step wave tail
        n_events = args.cpu_events or args.steps * args.batch
        cpu = reference_cpu_baseline(events, ncpu, n_events, budget_s=12.0)
        value = cpu["value"]
        line = dict(base)
        line["config"] = dict(config, events_per_step=args.batch,
                              reference_sample=f"{args.steps} steps of {args.batch} events, timed as one sustained "
                                               f"sample; a step is {args.batch} events")
        line.update({"impl": "reference", "value": value, "ms_per_step": 1e3 * args.batch / value,
                     "cpu_baseline": cpu,
                     "e2e": {"value": value, "unit": "events/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        import torch.distributed as tdist
        import datetime

        tdist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    events = generate(args.config, rank_first_event(rank, args.batch), args.batch, ncpu)
    res = (runner or run_ours)(args, rank, world, local, events)

    cpu = None
    if rank == 0 and world == 1 and runner is None:
        try:
            cpu = reference_cpu_baseline(events, ncpu, args.cpu_events or 2 * cpu_threads(ncpu), budget_s=12.0)
        except Exception as e:  # the CPU baseline is reported, not required
            cpu = {"value": None, "unit": "events/s", "cores": ncpu, "kind": "reference", "sample": f"failed: {e}"}

    if world > 1:
        import torch.distributed as tdist

        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        line = dict(base)
        line.update(res)
        line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
