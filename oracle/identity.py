"""Object-identity comparison of two LST event stores (test infrastructure).

``oracle/compare.py`` demands bit-identical stores.  This module answers the
looser question the stock-math reference needs: which objects exist on one
side and not on the other.  Every object is keyed by what it is made of,
never by its arena index (an index shifts inside a module as soon as one
object before it flips):

  md   (anchor hit, outer hit)                      MiniDoublet.h:193-266
  ls   the four hits of its two MDs                  Segment.h:358-390
  pls  pLS index with its isDup bits                 Segment.h:392-453, Kernels.h:384
  t3   its 6 hit indices                             Triplet.h:181-239
  t5   its 10 hit indices (+ isDup / TightCutFlag / partOfPT5)  Quintuplet.h:150-216
  pt3  (pLS index, 10 hit indices)                   PixelTriplet.h:134-204
  pt5  (pLS index, 14 hit indices)                   PixelTriplet.h:1961-2036
  tc   (type, pixel seed index, 14 hit slots)        TrackCandidate.h:111-163

An object present on one side only is a *root* flip when every constituent
it is built from (hits, MDs, LS, T3, T5, pLS) exists on the other side too,
with the same flags: the two sides then evaluated the same candidate and
decided differently.  Otherwise it is a *cascade* of a flip upstream.

Float values of objects present on both sides are compared as well: the
largest relative difference per field is reported.
"""
from __future__ import annotations

from collections import Counter

import numpy as np

from .compare import StoreIndex

STORES = ("md", "ls", "pls", "t3", "t5", "pt3", "pt5", "tc")

# Float fields compared (relative difference) on objects present on both sides.
VALUE_FIELDS = {
    "md": ("md.dphichanges", "md.dzs", "md.dphis", "md.anchorPhi", "md.anchorEta", "md.outerPhi", "md.outerEta"),
    "ls": ("ls.dPhis", "ls.dPhiChanges"),
    "t3": ("t3.betaIn", "t3.circleRadius"),
    "t5": ("t5.innerRadius", "t5.bridgeRadius", "t5.outerRadius", "t5.pt", "t5.eta", "t5.phi",
           "t5.score_rphisum", "t5.regressionRadius", "t5.rzChiSquared", "t5.chiSquared",
           "t5.nonAnchorChiSquared"),
    "pt3": ("pt3.pixelRadius", "pt3.tripletRadius", "pt3.pt", "pt3.eta", "pt3.phi", "pt3.score",
            "pt3.rPhiChiSquared", "pt3.rPhiChiSquaredInwards", "pt3.rzChiSquared"),
    "pt5": ("pt5.pixelRadius", "pt5.quintupletRadius", "pt5.score", "pt5.eta", "pt5.phi",
            "pt5.rzChiSquared", "pt5.rPhiChiSquared", "pt5.rPhiChiSquaredInwards"),
    "tc": ("tc.centerX", "tc.centerY", "tc.radius"),
}


class Objects:
    """The live objects of one side, keyed by identity.

    ``keys[store]`` is a list of tuples in arena order, ``index[store]`` the
    matching arena indices, ``parts[store]`` the constituent keys of each
    object as (store, key) pairs, and ``state[store]`` a per-object tuple of
    the flags that later stages set (dup marks, TightCutFlag)."""

    def __init__(self, get, n_lower: int, n_hits: int):
        self.get = get
        si = StoreIndex(get, n_lower, n_hits)
        self.si = si
        self.keys, self.index, self.parts, self.state = {}, {}, {}, {}

        a_hit = get("md.anchorHitIndices")
        o_hit = get("md.outerHitIndices")
        md_key = {int(i): (int(a_hit[i]), int(o_hit[i])) for i in si.md}
        self._put("md", si.md, [md_key[int(i)] for i in si.md], [() for _ in si.md])

        mdi = get("ls.mdIndices")
        ls_key, ls_parts = {}, {}
        for i in si.ls:
            i = int(i)
            m0, m1 = int(mdi[2 * i]), int(mdi[2 * i + 1])
            k0, k1 = md_key.get(m0, ("?", m0)), md_key.get(m1, ("?", m1))
            ls_key[i] = k0 + k1
            ls_parts[i] = (("md", k0), ("md", k1))
        self._put("ls", si.ls, [ls_key[int(i)] for i in si.ls], [ls_parts[int(i)] for i in si.ls])

        n_pls = min(si.n_pls, 50000)
        is_dup = get("ls.isDup")[:n_pls].astype(np.int64)
        part5 = get("ls.partOfPT5")[:n_pls].astype(np.int64)
        pls_keys = [(int(p),) for p in range(n_pls)]
        self._put("pls", np.arange(n_pls), pls_keys, [() for _ in range(n_pls)],
                  [(int(is_dup[p]), int(part5[p])) for p in range(n_pls)])

        h3 = get("t3.hitIndices")
        segi = get("t3.segmentIndices")
        t3_p5 = get("t3.partOfPT5")
        t3_key = {}
        t3_parts, t3_state = [], []
        for i in si.t3:
            i = int(i)
            t3_key[i] = tuple(int(x) for x in h3[6 * i: 6 * i + 6])
            s0, s1 = int(segi[2 * i]), int(segi[2 * i + 1])
            t3_parts.append((("ls", ls_key.get(s0, ("?", s0))), ("ls", ls_key.get(s1, ("?", s1)))))
            t3_state.append((int(t3_p5[i]),))
        self._put("t3", si.t3, [t3_key[int(i)] for i in si.t3], t3_parts, t3_state)

        h5 = get("t5.hitIndices")
        tri = get("t5.tripletIndices")
        dup5 = get("t5.isDup")
        tight = get("t5.TightCutFlag")
        t5_p5 = get("t5.partOfPT5")
        t5_key = {}
        t5_parts, t5_state = [], []
        for i in si.t5:
            i = int(i)
            t5_key[i] = tuple(int(x) for x in h5[10 * i: 10 * i + 10])
            a, b = int(tri[2 * i]), int(tri[2 * i + 1])
            t5_parts.append((("t3", t3_key.get(a, ("?", a))), ("t3", t3_key.get(b, ("?", b)))))
            t5_state.append((int(dup5[i]), int(tight[i]), int(t5_p5[i])))
        self._put("t5", si.t5, [t5_key[int(i)] for i in si.t5], t5_parts, t5_state)

        p3 = get("pt3.pixelSegmentIndices")
        h_p3 = get("pt3.hitIndices")
        tri3 = get("pt3.tripletIndices")
        dup_p3 = get("pt3.isDup")
        pls_base = int(get("ranges.segmentModuleIndices")[n_lower])
        pt3_key = {}
        pt3_parts, pt3_state = [], []
        for i in si.pt3:
            i = int(i)
            pls = int(p3[i]) - pls_base
            pt3_key[i] = (pls,) + tuple(int(x) for x in h_p3[10 * i: 10 * i + 10])
            t = int(tri3[i])
            pt3_parts.append((("pls", (pls,)), ("t3", t3_key.get(t, ("?", t)))))
            pt3_state.append((int(dup_p3[i]),))
        self._put("pt3", si.pt3, [pt3_key[int(i)] for i in si.pt3], pt3_parts, pt3_state)

        p5 = get("pt5.pixelIndices")
        h_p5 = get("pt5.hitIndices")
        t5i = get("pt5.T5Indices")
        dup_p5 = get("pt5.isDup")
        pt5_key = {}
        pt5_parts, pt5_state = [], []
        for i in si.pt5:
            i = int(i)
            pls = int(p5[i]) - pls_base
            pt5_key[i] = (pls,) + tuple(int(x) for x in h_p5[14 * i: 14 * i + 14])
            t = int(t5i[i])
            pt5_parts.append((("pls", (pls,)), ("t5", t5_key.get(t, ("?", t)))))
            pt5_state.append((int(dup_p5[i]),))
        self._put("pt5", si.pt5, [pt5_key[int(i)] for i in si.pt5], pt5_parts, pt5_state)

        typ = get("tc.trackCandidateType")
        seed = get("tc.pixelSeedIndex")
        htc = get("tc.hitIndices")
        direct = get("tc.directObjectIndices")
        tc_keys, tc_parts = [], []
        for i in si.tc:
            i = int(i)
            t = int(typ[i])
            tc_keys.append((t, int(seed[i])) + tuple(int(x) for x in htc[14 * i: 14 * i + 14]))
            d = int(direct[i])
            if t == 7:
                tc_parts.append((("pt5", pt5_key.get(d, ("?", d))),))
            elif t == 5:
                tc_parts.append((("pt3", pt3_key.get(d, ("?", d))),))
            elif t == 4:
                tc_parts.append((("t5", t5_key.get(d, ("?", d))),))
            else:  # type 8 stores the pLS index itself (TrackCandidate.h:521-525)
                tc_parts.append((("pls", (d,)),))
        self._put("tc", si.tc, tc_keys, tc_parts)

    def _put(self, store, index, keys, parts, state=None):
        self.index[store] = np.asarray(index, np.int64)
        self.keys[store] = keys
        self.parts[store] = parts
        self.state[store] = state if state is not None else [() for _ in keys]

    def key_set(self, store):
        return set(self.keys[store])

    def state_map(self):
        """{store: {key: flags}} over all stores (cached)."""
        if not hasattr(self, "_state_map"):
            self._state_map = {st: dict(zip(self.keys[st], self.state[st])) for st in STORES}
        return self._state_map


def diff(a: Objects, b: Objects, stores=STORES, max_examples: int = 20) -> dict:
    """Per store: objects only in a / only in b (multiset difference), how many
    of them are root flips, objects in both whose state flags differ, and the
    largest relative difference of each value field over the common objects."""
    out = {}
    for st in stores:
        ca, cb = Counter(a.keys[st]), Counter(b.keys[st])
        only_a = list((ca - cb).elements())
        only_b = list((cb - ca).elements())
        states = {"a": a.state_map(), "b": b.state_map()}
        pos_a = {k: j for j, k in enumerate(a.keys[st])}
        pos_b = {k: j for j, k in enumerate(b.keys[st])}

        def roots(only, side, other):
            pos = pos_a if side is a else pos_b
            mine, theirs = (states["a"], states["b"]) if side is a else (states["b"], states["a"])
            r = []
            for k in only:
                parts = side.parts[st][pos[k]]
                if all(pk in theirs[ps] and theirs[ps][pk] == mine[ps].get(pk) for ps, pk in parts):
                    r.append(k)
            return r

        root_a = roots(only_a, a, b)
        root_b = roots(only_b, b, a)
        state_diff = []
        common = [k for k in pos_a if k in pos_b]
        for k in common:
            sa, sb = a.state[st][pos_a[k]], b.state[st][pos_b[k]]
            if sa != sb:
                state_diff.append((k, sa, sb))
        values = {}
        if st in VALUE_FIELDS and common:
            ia = np.array([a.index[st][pos_a[k]] for k in common], np.int64)
            ib = np.array([b.index[st][pos_b[k]] for k in common], np.int64)
            for f in VALUE_FIELDS[st]:
                va, vb = a.get(f), b.get(f)
                if va is None or vb is None:
                    continue
                va = np.asarray(va, np.float64)[ia]
                vb = np.asarray(vb, np.float64)[ib]
                fin = np.isfinite(va) & np.isfinite(vb)
                same_nonfinite = ~fin & ((va == vb) | (np.isnan(va) & np.isnan(vb)))
                den = np.maximum(np.abs(va[fin]), np.abs(vb[fin]))
                rel = np.where(den > 0, np.abs(va[fin] - vb[fin]) / np.where(den > 0, den, 1), 0.0)
                values[f] = {"max_rel": float(rel.max()) if rel.size else 0.0,
                             "n_differ": int(np.count_nonzero(rel)) + int(np.count_nonzero(~fin & ~same_nonfinite)),
                             "n": int(va.size)}
        n = max(len(a.keys[st]), len(b.keys[st]), 1)
        out[st] = {
            "n_a": len(a.keys[st]), "n_b": len(b.keys[st]),
            "only_a": len(only_a), "only_b": len(only_b),
            "root_only_a": len(root_a), "root_only_b": len(root_b),
            "state_differ": len(state_diff),
            "flip_fraction": (len(only_a) + len(only_b) + len(state_diff)) / n,
            "root_fraction": (len(root_a) + len(root_b)) / n,
            "examples_root_a": root_a[:max_examples], "examples_root_b": root_b[:max_examples],
            "examples_state": state_diff[:max_examples],
            "values": values,
        }
    return out


def summary_line(d: dict) -> str:
    parts = []
    for st, r in d.items():
        parts.append(f"{st}: {r['n_a']}/{r['n_b']} -{r['only_a']}+{r['only_b']} (root {r['root_only_a']}+"
                     f"{r['root_only_b']}) state {r['state_differ']}")
    return "; ".join(parts)
