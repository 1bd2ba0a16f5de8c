"""Generates the golden fixtures of tests/golden/: known answers of the
reference CPU backend (oracle/_ref/liblstref_cr.so, built from the reference
sources) on seeded synthetic events.

ref_pins.json, the Event API: for each event a digest of the generator's
inputs, the reference's object counts after every stage, sha256 digests of
the live entries of the main object fields after the full chain
(oracle.compare.DIGEST_FIELDS), and for the single-muon events the complete
LST::getOutput hit lists.

seed_pins.json, the CMSSW entry point LST::run: for each event a digest of the
generator's CMSSW-layout seeds and hits, digests of the 23 vectors
LST::prepareInput produces, and digests of LST::run's outputs (hits, len,
seedIdx, trackCandidateType), with the complete outputs for the single-muon
events.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import compare, reflib  # noqa: E402
from tracklooper_b200 import gen  # noqa: E402
from tracklooper_b200.lst import STAGE_ORDER  # noqa: E402

EVENTS = [(1, i, 0.0) for i in range(4)] + [(2, 0, 0.0), (3, 0, 40.0)]
SEED_EVENTS = [(1, i, 0.0) for i in range(4)] + [(3, 1, 40.0), (2, 0, 0.0), (5, 0, 0.0)]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_pins.json")
SEED_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "seed_pins.json")

# element types of the compared fields (as in the CUDA library's field table)
DTYPES = {
    "hits.idxs": np.uint32,
    "md.anchorHitIndices": np.uint32, "md.outerHitIndices": np.uint32, "md.anchorPhi": np.float32,
    "md.nMDs": np.uint32, "ls.mdIndices": np.uint32, "ls.dPhiChanges": np.float32, "ls.nSegments": np.uint32,
    "t3.segmentIndices": np.uint32, "t3.betaIn": np.float32, "t3.nTriplets": np.uint32,
    "t5.tripletIndices": np.uint32, "t5.score_rphisum": np.float32, "t5.TightCutFlag": np.uint8,
    "t5.isDup": np.int8, "t5.nQuintuplets": np.uint32,
    "pt3.pixelSegmentIndices": np.uint32, "pt3.tripletIndices": np.uint32, "pt3.score": np.float32,
    "pt3.isDup": np.uint8, "pt3.nPixelTriplets": np.uint32,
    "pt5.pixelIndices": np.uint32, "pt5.T5Indices": np.uint32, "pt5.score": np.float32, "pt5.isDup": np.uint8,
    "pt5.nPixelQuintuplets": np.uint32,
    "tc.trackCandidateType": np.int16, "tc.hitIndices": np.uint32, "tc.pixelSeedIndex": np.int32,
    "tc.objectIndices": np.uint32, "tc.nTrackCandidates": np.uint32,
    "ranges.miniDoubletModuleIndices": np.int32, "ranges.segmentModuleIndices": np.int32,
    "ranges.tripletModuleIndices": np.int32, "ranges.quintupletModuleIndices": np.int32,
}


def input_digest(inp) -> str:
    h = hashlib.sha256()
    for a in (inp.x, inp.y, inp.z, inp.detId, inp.idxInNtuple):
        h.update(np.ascontiguousarray(a).tobytes())
    for k in sorted(inp.pls):
        h.update(np.ascontiguousarray(inp.pls[k]).tobytes())
    return h.hexdigest()[:32]


def stage_counts(get, n_lower):
    L = n_lower
    return {
        "md": int(get("md.nMDs")[:L].sum()),
        "ls": int(get("ls.nSegments")[:L].sum()),
        "pls": int(get("ls.nSegments")[L]),
        "t3": int(get("t3.nTriplets")[:L].sum()),
        "t5": int(get("t5.nQuintuplets")[:L].sum()),
        "pt5": int(get("pt5.nPixelQuintuplets")[0]),
        "pt3": int(get("pt3.nPixelTriplets")[0]),
        "tc": int(get("tc.nTrackCandidates")[0]),
    }


def output_lists(get):
    """LST::getOutput (SDL/LST.cc:367-427) on a store."""
    n = int(get("tc.nTrackCandidates")[0])
    types = get("tc.trackCandidateType")[:n]
    th = get("tc.hitIndices")
    idxs = get("hits.idxs")
    out = []
    for i in range(n):
        t = int(types[i])
        maxn = {7: 14, 5: 10, 4: 10, 8: 4}.get(t, 0)
        hits = []
        for k in range(maxn):
            g = int(th[14 * i + k])
            h = g if t == 8 else int(idxs[g])
            if t != 4 and len(hits) == 3 and hits[-1] == h:
                continue
            hits.append(h)
        out.append([t, hits])
    return out


def ref_getter(ref):
    def get(name):
        a = ref.field(name, dtype=DTYPES[name])
        return np.zeros(0, DTYPES[name]) if a is None else a
    return get


def pins_for(ref, inp):
    ref.reset()
    ref.add_inputs(inp)
    get = ref_getter(ref)
    counts = {}
    for st in STAGE_ORDER:
        ref.run_stage(st)
    counts = stage_counts(get, ref.n_lower)
    sizes = {"H": inp.n_hits, "MD": get("md.anchorHitIndices").size, "LS": get("ls.dPhiChanges").size,
             "T3": get("t3.betaIn").size, "T5": get("t5.score_rphisum").size}
    if sizes["T3"] == 0:
        sizes["T3"] = 1 << 40
    if sizes["T5"] == 0:
        sizes["T5"] = 1 << 40
    return counts, compare.store_digests(get, ref.n_lower, inp.n_hits, sizes), get


def array_digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()[:32]


def seed_digest(seeds) -> str:
    h = hashlib.sha256()
    for k in gen.SEED_FLOAT_FIELDS + ("see_q",):
        h.update(np.ascontiguousarray(seeds.see[k]).tobytes())
    for a in (seeds.hit_offsets, seeds.hit_idx, seeds.ph2_detId, seeds.ph2_x, seeds.ph2_y, seeds.ph2_z):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:32]


def seed_pins_for(ref, seeds, full_output: bool) -> dict:
    prep = ref.prepare_input(seeds)
    run = ref.run_lst(seeds)
    rec = {"n_seeds": seeds.n_seeds, "n_ph2": seeds.n_ph2, "inputs": seed_digest(seeds),
           "n_hits": int(prep["in_trkX_"].size), "n_pls": int(prep["in_ptIn_vec_"].size),
           "prepare": {k: array_digest(v) for k, v in sorted(prep.items())},
           "n_tc": int(run["len"].size), "run": {k: array_digest(v) for k, v in sorted(run.items())}}
    if full_output:
        bounds = np.concatenate(([0], np.cumsum(run["len"].astype(np.int64))))
        rec["output"] = [[int(run["trackCandidateType"][i]), int(run["seedIdx"][i]),
                          run["hits"][bounds[i]:bounds[i + 1]].tolist()] for i in range(run["len"].size)]
    return rec


def seed_main(ref):
    pins = {"reference": "liblstref_cr.so: SDL/LST.cc with ROOT's XYZVector restated (oracle/ref/shim/Math)",
            "events": []}
    for config, index, pileup in SEED_EVENTS:
        seeds = gen.generate_event(config, index, pileup).seeds
        rec = {"config": config, "index": index, "pileup": pileup}
        rec.update(seed_pins_for(ref, seeds, config == 1))
        pins["events"].append(rec)
        print("seeds", config, index, rec["n_pls"], rec["n_tc"])
    with open(SEED_OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", SEED_OUT)


def main():
    ref = reflib.RefLST("cr")
    seed_main(ref)
    pins = {"reference": "liblstref_cr.so (strict IEEE, double-rounded float transcendentals, T5 DNN)",
            "events": []}
    for config, index, pileup in EVENTS:
        inp = gen.generate_event(config, index, pileup)
        counts, digests, get = pins_for(ref, inp)
        rec = {"config": config, "index": index, "pileup": pileup, "n_hits": inp.n_hits, "n_pls": inp.n_pls,
               "inputs": input_digest(inp), "counts": counts, "digests": digests}
        if config == 1:
            rec["output"] = output_lists(get)
        pins["events"].append(rec)
        print(config, index, counts)
    ref.close()
    with open(OUT, "w") as f:
        json.dump(pins, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
