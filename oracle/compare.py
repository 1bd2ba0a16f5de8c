"""Field-by-field comparison of two LST event stores (test infrastructure).

Both sides expose ``get(name) -> numpy array`` over the reference's store and
field names (``md.anchorHitIndices``, ``t5.score_rphisum``, ...): the reference
CPU backend through oracle/reflib.py and the CUDA path through
tracklooper_b200.lst.  Objects live at per-module offsets inside fixed-size
arenas, so only the live slots are compared: for each store the valid
indices are rebuilt from that side's own range arrays and counts, which are
compared first.  Floats are compared bit for bit.

Which fields each reference store function writes (and so which are
comparable) follows SDL/MiniDoublet.h:193-266, SDL/Segment.h:358-453,
SDL/Triplet.h:181-239, SDL/Quintuplet.h:150-216, SDL/PixelTriplet.h:134-204
and :1961-2036, SDL/TrackCandidate.h:111-163.
"""
from __future__ import annotations

import numpy as np

N_PLS_MAX = 50000

# Fields the reference never writes for some objects (left as allocated).
SKIP_ALWAYS = {
    "pt3.pixelRadiusError",  # not stored by addPixelTripletToMemory
    "pt3.partOfPT5",  # not stored by addPixelTripletToMemory
}
# Segment fields addPixelSegmentToMemory does not write for pixel segments.
PLS_UNSET = {"ls.dPhis", "ls.dPhiMins", "ls.dPhiMaxs", "ls.dPhiChangeMins", "ls.dPhiChangeMaxs"}
# Track-candidate fields addpLSTrackCandidateToMemory does not write (type 8).
TC_PLS_UNSET = {"tc.logicalLayers", "tc.lowerModuleIndices", "tc.centerX", "tc.centerY", "tc.radius"}

STAGE_STORES = {
    "md": ("hits", "md"),
    "ls": ("ls",),
    "t3": ("t3",),
    "t5": ("t5",),
    "pls_clean": ("ls",),
    "pt5": ("pt5", "tc"),
    "pt3": ("pt3",),
    "tc": ("tc",),
}


def _ranges(starts, counts):
    starts = np.asarray(starts, np.int64)
    counts = np.asarray(counts, np.int64)
    keep = counts > 0
    starts, counts = starts[keep], counts[keep]
    if counts.size == 0:
        return np.zeros(0, np.int64)
    total = int(counts.sum())
    idx = np.repeat(starts - np.concatenate(([0], np.cumsum(counts)[:-1])), counts) + np.arange(total)
    return idx


def _expand(idx, mult):
    if mult == 1:
        return idx
    return (idx[:, None] * mult + np.arange(mult)[None, :]).ravel()


class StoreIndex:
    """Valid object indices of every store of one side."""

    def __init__(self, get, n_lower: int, n_hits: int):
        self.get = get
        L = n_lower
        rg_md = get("ranges.miniDoubletModuleIndices")
        nmd = get("md.nMDs")
        self.md = _ranges(rg_md[: L + 1], nmd[: L + 1])
        self.md_pixel = _ranges(rg_md[L:L + 1], nmd[L:L + 1])
        rg_ls = get("ranges.segmentModuleIndices")
        nls = get("ls.nSegments")
        self.ls = _ranges(rg_ls[:L], nls[:L])
        self.ls_pixel = _ranges(rg_ls[L:L + 1], nls[L:L + 1])
        self.n_pls = int(nls[L])
        self.pls = np.arange(min(self.n_pls, N_PLS_MAX))
        rg_t3 = get("ranges.tripletModuleIndices")
        nt3 = get("t3.nTriplets")
        self.t3 = _ranges(rg_t3[:L], nt3[:L])
        rg_t5 = get("ranges.quintupletModuleIndices")
        nt5 = get("t5.nQuintuplets")
        ok = rg_t5[:L] != -1
        self.t5 = _ranges(rg_t5[:L][ok], nt5[:L][ok])
        self.pt3 = np.arange(int(get("pt3.nPixelTriplets")[0]))
        self.pt5 = np.arange(int(get("pt5.nPixelQuintuplets")[0]))
        self.n_tc = int(get("tc.nTrackCandidates")[0])
        self.tc = np.arange(self.n_tc)
        self.hits = np.arange(n_hits)


def _object_index(store: str, name: str, arr_len: int, si: StoreIndex, sizes: dict):
    """(indices, multiplicity) of the live entries of field `name`, or None to compare all."""
    fld = name.split(".", 1)[1]
    if name == "ranges.indicesOfEligibleT5Modules":
        return np.arange(int(si.get("ranges.nEligibleT5Modules")[0])), 1
    if store == "hits":
        if arr_len % sizes["H"] == 0 and arr_len // sizes["H"] <= 1 and not fld.startswith("hitRanges"):
            return si.hits, 1
        return None
    if store == "md":
        if arr_len >= sizes["MD"] and arr_len % sizes["MD"] == 0:
            return si.md, arr_len // sizes["MD"]
        return None
    if store == "ls":
        if arr_len >= sizes["LS"] and arr_len % sizes["LS"] == 0:
            idx = si.ls if name in PLS_UNSET else np.concatenate([si.ls, si.ls_pixel])
            return idx, arr_len // sizes["LS"]
        if arr_len >= N_PLS_MAX and arr_len % N_PLS_MAX == 0:
            return si.pls, arr_len // N_PLS_MAX
        return None
    if store == "t3":
        if arr_len >= sizes["T3"] and arr_len % sizes["T3"] == 0:
            return si.t3, arr_len // sizes["T3"]
        return None
    if store == "t5":
        if arr_len >= sizes["T5"] and arr_len % sizes["T5"] == 0:
            return si.t5, arr_len // sizes["T5"]
        return None
    if store in ("pt3", "pt5", "tc"):
        cap = {"pt3": 5000, "pt5": 15000, "tc": 31000}[store]
        if arr_len >= cap and arr_len % cap == 0:
            idx = {"pt3": si.pt3, "pt5": si.pt5, "tc": si.tc}[store]
            if store == "tc" and name in TC_PLS_UNSET:
                types = si.get("tc.trackCandidateType")[: si.n_tc]
                idx = idx[types != 8]
            return idx, arr_len // cap
        return None
    return None


def compare_stores(get_a, get_b, names, n_lower: int, n_hits: int, sizes: dict, max_report: int = 5):
    """Compares the given fields; returns a list of human-readable mismatch lines.

    get_a is the side whose range arrays define the live objects (both sides'
    counts are compared first, so after that they agree)."""
    problems = []
    sa = StoreIndex(get_a, n_lower, n_hits)
    for name in names:
        if name in SKIP_ALWAYS:
            continue
        a = get_a(name)
        b = get_b(name)
        if a is None:
            problems.append(f"{name}: missing")
            continue
        if b is None:  # a store the other side allocated with zero length
            b = np.zeros(0, a.dtype)
        store = name.split(".", 1)[0]
        sel = _object_index(store, name, a.size, sa, sizes)
        if sel is None:
            n = min(a.size, b.size)
            av, bv = a[:n], b[:n]
            where = np.arange(n)
        else:
            idx, mult = sel
            full = _expand(idx, mult)
            if full.size and int(full.max()) >= min(a.size, b.size):
                problems.append(f"{name}: live entries up to {int(full.max())} but lengths {a.size}, {b.size}")
                continue
            av, bv, where = a[full], b[full], full
        if av.dtype.kind == "f":
            av = av.view(np.uint32 if av.dtype.itemsize == 4 else np.uint64)
            bv = np.ascontiguousarray(bv).view(av.dtype)
        else:
            bv = bv.astype(av.dtype, copy=False)
        bad = np.nonzero(av != bv)[0]
        if bad.size:
            ex = ", ".join(f"[{int(where[i])}] {a[where[i]]!r} vs {b[where[i]]!r}" for i in bad[:max_report])
            problems.append(f"{name}: {bad.size}/{av.size} differ: {ex}")
    return problems


def stage_fields(all_names, stages):
    stores = set()
    for st in stages:
        stores.update(STAGE_STORES[st])
    return [n for n in all_names if n.split(".", 1)[0] in stores or n.startswith("ranges.")]


# Fields whose live entries are digested for the golden fixtures: every
# object's identity (its hits / constituents) and one float per object type.
DIGEST_FIELDS = (
    "md.anchorHitIndices", "md.outerHitIndices", "md.anchorPhi",
    "ls.mdIndices", "ls.dPhiChanges",
    "t3.segmentIndices", "t3.betaIn",
    "t5.tripletIndices", "t5.score_rphisum", "t5.TightCutFlag", "t5.isDup",
    "pt3.pixelSegmentIndices", "pt3.tripletIndices", "pt3.score", "pt3.isDup",
    "pt5.pixelIndices", "pt5.T5Indices", "pt5.score", "pt5.isDup",
    "tc.trackCandidateType", "tc.hitIndices", "tc.pixelSeedIndex", "tc.objectIndices",
)


def store_digests(get, n_lower: int, n_hits: int, sizes: dict) -> dict:
    """sha256 of the live entries of DIGEST_FIELDS (bit patterns for floats)."""
    import hashlib

    si = StoreIndex(get, n_lower, n_hits)
    out = {}
    for name in DIGEST_FIELDS:
        a = get(name)
        store = name.split(".", 1)[0]
        sel = _object_index(store, name, a.size, si, sizes)
        if sel is None:
            v = a
        else:
            idx, mult = sel
            v = a[_expand(idx, mult)]
        out[name] = hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()[:32]
    return out
