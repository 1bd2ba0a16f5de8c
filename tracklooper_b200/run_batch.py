"""Runs a batch of seeded synthetic events through the CUDA chain and prints
per-event object counts and the batch time.

  python -m tracklooper_b200.run_batch --config 2 --events 8 [--repeat 3] [--cuts] [--tune-cache PATH]

--config selects the generator configuration (1 muon gun, 2 PU200-shaped,
3 PU140-250, 5 PU250 with displaced tracks); the events are generated with
seeds (config << 32) | index, uploaded packed, and run once per --repeat.
With --tune-cache the launch shapes come from the autotuner's cache for this
geometry, device, batch size and build, or from a sweep that is then stored
there (lst_autotune_load / lst_autotune).
"""
from __future__ import annotations

import argparse
import json
import time
from concurrent.futures import ThreadPoolExecutor

from . import gen, lst


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--events", type=int, default=8)
    ap.add_argument("--first", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--cuts", action="store_true", help="cut-only T5 selection instead of the DNN")
    ap.add_argument("--json", action="store_true")
    ap.add_argument("--tune-cache", default=None, help="autotuner cache file (load, or sweep and store)")
    args = ap.parse_args(argv)

    with ThreadPoolExecutor(max_workers=16) as pool:
        inputs = list(pool.map(lambda i: gen.generate_event(args.config, args.first + i), range(args.events)))
    es = lst.ES(device=args.device)
    eset = lst.EventSet(es, n_slots=args.events, max_hits=max(i.n_hits for i in inputs) + 1024)
    if args.cuts:
        eset.set_t5_method(lst.T5_CUTS)
    blob, offsets = lst.pack_events(inputs)
    if args.tune_cache:
        if not eset.autotune_load(args.events, args.tune_cache):
            eset.upload_packed(0, blob, offsets)
            eset.autotune(0, args.events, args.tune_cache)
    times = []
    for r in range(args.repeat):
        t0 = time.perf_counter()
        if r == 0:
            eset.upload_packed(0, blob, offsets)
        else:
            eset.ingest(0, args.events)
        eset.run(0, args.events)
        eset.sync()
        times.append(time.perf_counter() - t0)
    counts = eset.batch_counts(0, args.events)
    keys = ("nHits", "nPixelSegments", "nMiniDoublets", "nSegments", "nTriplets", "nQuintuplets",
            "nPixelQuintuplets", "nPixelTriplets", "nTrackCandidates", "status")
    if args.json:
        print(json.dumps({"times_s": times, "counts": [{k: c[k] for k in keys} for c in counts]}))
    else:
        for i, c in enumerate(counts):
            print(f"event {args.first + i}: " + " ".join(f"{k}={c[k]}" for k in keys))
        print(f"batch of {args.events}: " + ", ".join(f"{t * 1e3:.1f} ms" for t in times))
    eset.close()
    es.close()


if __name__ == "__main__":
    main()
