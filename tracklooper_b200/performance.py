"""Track-candidate efficiency, fake rate and duplicate rate from simulation
truth, with the reference's definitions:

* a track candidate is matched to a simulated particle when strictly more
  than 75% of its distinct hits come from that particle
  (code/core/trkCore.cc:231-403, matchedSimTrkIdxs; one particle per hit
  here, -1 for noise), and is a fake when it matches none
  (code/core/write_sdl_ntuple.cc:873-874);
* a track candidate is a duplicate when the particle it matches is matched
  by more than one candidate (code/core/write_sdl_ntuple.cc:284-300);
* the efficiency of a set of particles is the fraction matched by at least
  one candidate (sim_TC_matched > 0, efficiency/src/performance.cc:44-80),
  per candidate type through the type mask (sim_TC_matched_mask); the fake
  and duplicate rates are fractions of the candidates
  (efficiency/src/performance.cc:130, :219).

The candidates are read from an event's track-candidate store
(trackCandidateType, hitIndices, directObjectIndices; SDL/TrackCandidate.h:
111-163), the truth from the generator's per-hit particle index.  The
reference's denominators are hard-scatter particles (sim_event == 0,
write_sdl_ntuple.cc:213-218); the seeded events mark no such flag, so the
hard process is taken as the leading particles that share the first
particle's production vertex (the generator emits them first), and the
pileup particles are reported as a second set.
"""
from __future__ import annotations

import numpy as np

TYPE_NAMES = {7: "pT5", 5: "pT3", 4: "T5", 8: "pLS"}


def tc_hits(types: np.ndarray, hit_slots: np.ndarray, direct: np.ndarray, pls_hits: np.ndarray) -> list:
    """Event-local hit indices of each candidate.  Types 7, 5 and 4 store
    them in their 14 / 10 slots; a pLS candidate (type 8) stores its pixel
    hits' ntuple indices, so its hits come from its pLS (direct index) in
    pls_hits (n_pls, 4)."""
    out = []
    for i, t in enumerate(types):
        t = int(t)
        if t == 8:
            out.append(np.asarray(pls_hits[int(direct[i])], np.int64))
        else:
            n = {7: 14, 5: 10, 4: 10}.get(t, 0)
            out.append(np.asarray(hit_slots[14 * i: 14 * i + n], np.int64))
    return out


def match(hits_per_tc: list, hit_sim: np.ndarray) -> np.ndarray:
    """The particle each candidate matches, -1 for a fake."""
    sim = np.asarray(hit_sim, np.int64)
    out = np.full(len(hits_per_tc), -1, np.int64)
    for i, h in enumerate(hits_per_tc):
        u = np.unique(h)
        if u.size == 0:
            continue
        s = sim[u]
        vals, cnt = np.unique(s, return_counts=True)
        k = int(np.argmax(cnt))
        if vals[k] >= 0 and cnt[k] > 0.75 * u.size:
            out[i] = vals[k]
    return out


def hard_process(particles: np.ndarray) -> np.ndarray:
    """Mask of the hard-process particles: the leading run that shares the
    first particle's production vertex."""
    n = particles.shape[0]
    mask = np.zeros(n, bool)
    if n == 0:
        return mask
    v0 = particles[0, 4:7]
    for i in range(n):
        if not np.array_equal(particles[i, 4:7], v0):
            break
        mask[i] = True
    return mask


def event_performance(types, hit_slots, direct, pls_hits, hit_sim, particles, pt_min: float = 1.0,
                      eta_max: float = 2.4) -> dict:
    """Counts of one event (summable over events with ``combine``)."""
    types = np.asarray(types)
    hits = tc_hits(types, np.asarray(hit_slots), np.asarray(direct), np.asarray(pls_hits))
    m = match(hits, hit_sim)
    n_part = particles.shape[0]
    matched_by = np.bincount(m[m >= 0], minlength=n_part) if n_part else np.zeros(0, np.int64)
    type_mask = np.zeros(n_part, np.int64)
    for t, s in zip(types, m):
        if s >= 0:
            type_mask[s] |= 1 << int(t)
    dup = np.array([s >= 0 and matched_by[s] > 1 for s in m], bool)
    pt, eta = particles[:, 0], particles[:, 1]
    sel = (pt > pt_min) & (np.abs(eta) < eta_max) & (particles[:, 3] != 0)
    hard = hard_process(particles)
    res = {"tc": int(types.size), "fake": int(np.sum(m < 0)), "duplicate": int(dup.sum()), "by_type": {}}
    for t, name in TYPE_NAMES.items():
        sel_t = types == t
        res["by_type"][name] = {"tc": int(sel_t.sum()), "fake": int(np.sum(sel_t & (m < 0))),
                                "duplicate": int(np.sum(sel_t & dup))}
    for set_name, pmask in (("hard", sel & hard), ("pileup", sel & ~hard)):
        res[set_name] = {"particles": int(pmask.sum()), "matched": int(np.sum(pmask & (matched_by > 0))),
                         "matched_by_type": {name: int(np.sum(pmask & ((type_mask >> t) & 1 == 1)))
                                             for t, name in TYPE_NAMES.items()}}
    return res


def combine(events: list) -> dict:
    """Sums event counts and forms the rates."""
    out = {"events": len(events), "tc": 0, "fake": 0, "duplicate": 0,
           "by_type": {n: {"tc": 0, "fake": 0, "duplicate": 0} for n in TYPE_NAMES.values()},
           "hard": {"particles": 0, "matched": 0, "matched_by_type": {n: 0 for n in TYPE_NAMES.values()}},
           "pileup": {"particles": 0, "matched": 0, "matched_by_type": {n: 0 for n in TYPE_NAMES.values()}}}
    for e in events:
        for k in ("tc", "fake", "duplicate"):
            out[k] += e[k]
        for n in TYPE_NAMES.values():
            for k in ("tc", "fake", "duplicate"):
                out["by_type"][n][k] += e["by_type"][n][k]
        for s in ("hard", "pileup"):
            out[s]["particles"] += e[s]["particles"]
            out[s]["matched"] += e[s]["matched"]
            for n in TYPE_NAMES.values():
                out[s]["matched_by_type"][n] += e[s]["matched_by_type"][n]
    out["fake_rate"] = out["fake"] / max(out["tc"], 1)
    out["duplicate_rate"] = out["duplicate"] / max(out["tc"], 1)
    for n, b in out["by_type"].items():
        b["fake_rate"] = b["fake"] / max(b["tc"], 1)
        b["duplicate_rate"] = b["duplicate"] / max(b["tc"], 1)
    for s in ("hard", "pileup"):
        out[s]["efficiency"] = out[s]["matched"] / max(out[s]["particles"], 1)
    return out


def from_store(get, inp, pt_min: float = 1.0, eta_max: float = 2.4) -> dict:
    """event_performance of one event whose stores `get(name)` reads (the
    CUDA path's lst.Event.field, an EventSet slot, or the reference's)."""
    n = int(get("tc.nTrackCandidates")[0])
    pls_hits = np.stack([inp.pls[f"hitIndices{k}"] for k in range(4)], axis=1) if inp.n_pls else np.zeros((0, 4))
    return event_performance(get("tc.trackCandidateType")[:n], get("tc.hitIndices")[:14 * n],
                             get("tc.directObjectIndices")[:n], pls_hits, inp.hit_sim, inp.particles, pt_min, eta_max)
