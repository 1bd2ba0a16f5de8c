"""Cut-flip tracer and FP64 re-evaluation oracle (test infrastructure).

``Tracer`` drives oracle/_ref/liblsttrace.so (oracle/trace/lst_trace.cc),
which rebuilds one object from its hits in three arithmetics:

  MODE_CR     IEEE single precision, transcendentals float(f(double(x)))
              -- the arithmetic of the CUDA path and of the parity oracle;
  MODE_GLIBC  IEEE single precision, glibc's float transcendentals -- the
              arithmetic of the reference's stock CPU backend;
  MODE_F64    the same formulas in double precision from the same float
              inputs -- the FP64 re-evaluation.

``trace_flip`` takes an object that one single-precision build keeps and
the other does not, finds the first comparison of its selection whose
outcome differs between MODE_CR and MODE_GLIBC, and reports the comparison's
source line, its operands in all three arithmetics and the distance of the
operand from its threshold: in float ulps of the threshold, and relative to
the single-precision rounding error of the margin (the flip is a rounding
effect when the exact margin is smaller than that error).

``values`` returns an object's stored floats (pt, eta, phi, radii, chi2,
scores) in any of the arithmetics, for the FP64 comparison of the stored
outputs.
"""
from __future__ import annotations

import ctypes
import functools
import os
import subprocess

import numpy as np

from . import reflib

MODE_CR, MODE_GLIBC, MODE_F64 = 0, 1, 2
KINDS = {"md": 0, "ls": 1, "t3": 2, "t5": 3, "pt3": 4, "pt5": 5}
OPS = {0: "<", 1: "<=", 2: ">", 3: ">=", 4: "==", 5: "!="}

# The stored floats lsttr_eval returns per kind, in order.
VALUE_NAMES = {
    "md": ("dzs", "dphis", "dphichanges", "noShiftedDzs", "noShiftedDphis", "noShiftedDphiChanges",
           "shiftedXs", "shiftedYs", "shiftedZs"),
    "ls": ("dPhis", "dPhiMins", "dPhiMaxs", "dPhiChanges", "dPhiChangeMins", "dPhiChangeMaxs"),
    "t3": ("betaIn", "circleRadius", "circleCenterX", "circleCenterY"),
    "t5": ("innerRadius", "bridgeRadius", "outerRadius", "pt", "eta", "phi", "score_rphisum", "regressionRadius",
           "regressionG", "regressionF", "rzChiSquared", "chiSquared", "nonAnchorChiSquared", "dnnScore",
           "TightCutFlag"),
    "pt3": ("pixelRadius", "pixelRadiusError", "tripletRadius", "pt", "eta", "phi", "eta_pix", "phi_pix", "score",
            "rPhiChiSquared", "rPhiChiSquaredInwards", "rzChiSquared"),
    "pt5": ("pixelRadius", "quintupletRadius", "score", "eta", "phi", "centerX", "centerY", "rzChiSquared",
            "rPhiChiSquared", "rPhiChiSquaredInwards"),
}


class Rec(ctypes.Structure):
    _fields_ = [("site", ctypes.c_void_p), ("lhs", ctypes.c_double), ("rhs", ctypes.c_double), ("op", ctypes.c_int),
                ("result", ctypes.c_int)]


def library_path() -> str:
    return os.path.join(reflib.REF_DIR, "liblsttrace.so")


def available() -> bool:
    return os.path.exists(library_path())


def ulp32(x: float) -> float:
    """Spacing of IEEE single-precision numbers at |x|."""
    return float(np.spacing(np.float32(abs(x)))) if np.isfinite(x) else float("nan")


class Tracer:
    def __init__(self, weights: np.ndarray | None = None, wp: float | None = None, geometry_dir: str | None = None):
        from tracklooper_b200 import geometry, t5dnn

        path = library_path()
        if not os.path.exists(path):
            raise FileNotFoundError(f"tracer library not built: {path}")
        lib = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        lib.lsttr_create.restype = vp
        lib.lsttr_create.argtypes = [ctypes.c_char_p, vp, ctypes.c_float]
        lib.lsttr_destroy.argtypes = [vp]
        lib.lsttr_set_hits.argtypes = [vp, ctypes.c_uint] + [vp] * 5
        lib.lsttr_set_pls.argtypes = [vp, ctypes.c_uint] + [vp] * 18
        lib.lsttr_eval.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp, ctypes.c_int,
                                   ctypes.POINTER(ctypes.c_int), vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_uint)]
        lib.lsttr_site_offset.restype = ctypes.c_ulonglong
        lib.lsttr_site_offset.argtypes = [vp]
        self.lib = lib
        w = np.ascontiguousarray(t5dnn.reference_weights() if weights is None else weights, np.float32).ravel()
        wp = t5dnn.REFERENCE_WP if wp is None else wp
        self.h = lib.lsttr_create((geometry_dir or geometry.geometry_dir()).encode(), w.ctypes.data, float(wp))
        if not self.h:
            raise RuntimeError("tracer failed to load the event setup")
        self._keep = []

    def close(self):
        if self.h:
            self.lib.lsttr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_event(self, inp):
        from tracklooper_b200.gen import PLS_FIELDS

        keep = []

        def p(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            keep.append(a)
            return a.ctypes.data

        self.lib.lsttr_set_hits(self.h, inp.n_hits, p(inp.x, np.float32), p(inp.y, np.float32), p(inp.z, np.float32),
                                p(inp.detId, np.uint32), p(inp.idxInNtuple, np.uint32))
        self.lib.lsttr_set_pls(self.h, inp.n_pls, *[p(inp.pls[name], dt) for name, dt in PLS_FIELDS])

    def eval(self, store: str, key, mode: int, use_dnn: bool = True):
        """(passes, {value name: value}, [trace records], constituent-fail bits)."""
        k = np.ascontiguousarray(key, np.uint32)
        vals = np.zeros(32, np.float64)
        nv = ctypes.c_int()
        cap = 4096
        tr = (Rec * cap)()
        nt = ctypes.c_int()
        fail = ctypes.c_uint()
        rc = self.lib.lsttr_eval(self.h, mode, KINDS[store], int(use_dnn), k.ctypes.data, k.size, vals.ctypes.data,
                                 vals.size, ctypes.byref(nv), tr, cap, ctypes.byref(nt), ctypes.byref(fail))
        if rc < 0:
            raise ValueError(f"malformed {store} key {tuple(key)}")
        names = VALUE_NAMES[store]
        values = {n: float(vals[i]) for i, n in enumerate(names[: nv.value])}
        trace = [(tr[i].site, tr[i].lhs, tr[i].rhs, tr[i].op, tr[i].result) for i in range(min(nt.value, cap))]
        return bool(rc), values, trace, int(fail.value)

    def values(self, store: str, key, mode: int = MODE_F64, use_dnn: bool = True) -> dict:
        return self.eval(store, key, mode, use_dnn)[1]

    @functools.lru_cache(maxsize=4096)
    def site(self, addr: int) -> str:
        """file:line (function) of a comparison's code address."""
        off = int(self.lib.lsttr_site_offset(ctypes.c_void_p(addr)))
        if not off:
            return "?"
        try:
            out = subprocess.run(["addr2line", "-e", library_path(), "-f", "-C", "-i", hex(off - 1)],
                                 capture_output=True, text=True, timeout=30).stdout.split("\n")
        except (OSError, subprocess.TimeoutExpired):
            return hex(off)
        func, loc = (out + ["", ""])[:2]
        loc = loc.split(" (discriminator")[0]
        parts = loc.split("/")
        short = "/".join(parts[-2:]) if len(parts) >= 2 else loc
        return f"{short} ({func.split('(')[0]})"

    def trace_flip(self, store: str, key, use_dnn: bool = True) -> dict:
        """The comparison that decides the object differently in the two
        single-precision arithmetics, with its operands in all three."""
        p_cr, v_cr, t_cr, f_cr = self.eval(store, key, MODE_CR, use_dnn)
        p_gl, v_gl, t_gl, f_gl = self.eval(store, key, MODE_GLIBC, use_dnn)
        p_64, v_64, t_64, f_64 = self.eval(store, key, MODE_F64, use_dnn)
        out = {"store": store, "key": [int(x) for x in key], "pass_cr": p_cr, "pass_glibc": p_gl, "pass_f64": p_64,
               "constituents_fail_cr": f_cr, "constituents_fail_glibc": f_gl, "explained": False}
        if f_cr != f_gl:
            out["reason"] = "a constituent is decided differently"
            return out
        if p_cr == p_gl:
            out["reason"] = "same decision in both single-precision arithmetics"
            return out
        n = min(len(t_cr), len(t_gl))
        i = next((j for j in range(n) if t_cr[j][4] != t_gl[j][4] or t_cr[j][0] != t_gl[j][0]), None)
        if i is None or t_cr[i][0] != t_gl[i][0]:
            out["reason"] = "the two traces part before a differing comparison"
            return out
        site, lc, rc_, op, _ = t_cr[i]
        _, lg, rg, _, _ = t_gl[i]
        same_path_64 = i < len(t_64) and t_64[i][0] == site and all(t_64[j][4] == t_cr[j][4] for j in range(i))
        l64, r64 = (t_64[i][1], t_64[i][2]) if same_path_64 else (float("nan"), float("nan"))
        d_cr, d_gl, d_64 = lc - rc_, lg - rg, l64 - r64
        scale = ulp32(r64 if np.isfinite(r64) else rc_)
        err = max(abs(d_cr - d_64), abs(d_gl - d_64)) if np.isfinite(d_64) else float("nan")
        out.update({
            "site": self.site(site), "op": OPS.get(op, "?"),
            "lhs": {"cr": lc, "glibc": lg, "f64": l64}, "rhs": {"cr": rc_, "glibc": rg, "f64": r64},
            "margin_ulps": {"cr": abs(d_cr) / scale, "glibc": abs(d_gl) / scale,
                            "f64": abs(d_64) / scale if np.isfinite(d_64) else None},
            "margin_over_rounding_error": (abs(d_64) / err) if np.isfinite(d_64) and err > 0 else None,
            "comparison_index": i,
        })
        # A rounding-level flip: the exact margin is within the single-precision
        # error of the margin on the two sides (the threshold lies inside the
        # band the two rounded operands span).
        out["explained"] = bool(np.isfinite(d_64) and abs(d_64) <= err)
        return out


def _t5_pair_comparisons(v1: dict, v2: dict, f32: bool):
    """The comparisons the two T5 duplicate-removal passes take for a pair
    (SDL/Kernels.h:202-320): (label, lhs, rhs, outcome), in order, with
    float arithmetic where f32 (the stored values are floats) else double."""
    t = np.float32 if f32 else np.float64
    e1, p1, s1 = t(v1["eta"]), t(v1["phi"]), t(v1["score_rphisum"])
    e2, p2, s2 = t(v2["eta"]), t(v2["phi"]), t(v2["score_rphisum"])
    pi = t(np.float32(np.pi))
    d_eta = abs(t(e1 - e2))
    d_phi = t(p1 - p2)
    if d_phi > pi:
        d_phi = t(d_phi - t(2) * pi)
    elif d_phi < -pi:
        d_phi = t(d_phi + t(2) * pi)
    d_r2 = t(t(d_eta * d_eta) + t(d_phi * d_phi))
    c01, c001 = float(np.float32(0.1)), float(np.float32(0.001))
    return [("dEta > 0.1", float(d_eta), c01, bool(d_eta > c01)),
            ("|dPhi| > 0.1", float(abs(d_phi)), c01, bool(abs(d_phi) > c01)),
            ("dR2 < 0.001", float(d_r2), c001, bool(d_r2 < c001)),
            ("score1 >= score2", float(s1), float(s2), bool(s1 >= s2)),
            ("score1 > score2", float(s1), float(s2), bool(s1 > s2)),
            ("score1 < score2", float(s1), float(s2), bool(s1 < s2))]


def trace_t5_state(tr: Tracer, key, partners, use_dnn: bool = True) -> dict:
    """Explains a T5 whose duplicate flag differs between the two
    single-precision arithmetics: among the T5s sharing at least five hits
    with it (partners), the first pair whose duplicate-removal comparisons
    come out differently, with the margins of that comparison."""
    key = tuple(int(x) for x in key)
    v = {m: tr.values("t5", key, m, use_dnn) for m in (MODE_CR, MODE_GLIBC, MODE_F64)}
    out = {"store": "t5", "key": list(key), "kind": "duplicate flag", "explained": False}
    for pk in partners:
        pk = tuple(int(x) for x in pk)
        w = {m: tr.values("t5", pk, m, use_dnn) for m in (MODE_CR, MODE_GLIBC, MODE_F64)}
        c_cr = _t5_pair_comparisons(v[MODE_CR], w[MODE_CR], True)
        c_gl = _t5_pair_comparisons(v[MODE_GLIBC], w[MODE_GLIBC], True)
        c_64 = _t5_pair_comparisons(v[MODE_F64], w[MODE_F64], False)
        for (lab, lc, rc_, oc), (_, lg, rg, og), (_, l64, r64, _) in zip(c_cr, c_gl, c_64):
            if oc == og:
                continue
            d_cr, d_gl, d_64 = lc - rc_, lg - rg, l64 - r64
            scale = ulp32(r64)
            err = max(abs(d_cr - d_64), abs(d_gl - d_64))
            out.update({"partner": list(pk), "site": "T5 duplicate removal (SDL/Kernels.h:202-320)", "op": lab,
                        "lhs": {"cr": lc, "glibc": lg, "f64": l64}, "rhs": {"cr": rc_, "glibc": rg, "f64": r64},
                        "margin_ulps": {"cr": abs(d_cr) / scale, "glibc": abs(d_gl) / scale,
                                        "f64": abs(d_64) / scale},
                        "margin_over_rounding_error": abs(d_64) / err if err > 0 else None,
                        "explained": bool(abs(d_64) <= err)})
            return out
    out["reason"] = "no partner whose comparisons differ"
    return out


def shared_hits(a, b) -> int:
    """Hits two objects have in common (as multisets)."""
    from collections import Counter

    return sum((Counter(a) & Counter(b)).values())


# Per store: (count field, occupancy field, module of an object) for the
# occupancy-cap check.
_CAP_FIELDS = {
    "md": ("md.nMDs", "md.totOccupancyMDs", "md.moduleIndices"),
    "ls": ("ls.nSegments", "ls.totOccupancySegments", "ls.innerLowerModuleIndices"),
    "t3": ("t3.nTriplets", "t3.totOccupancyTriplets", "t3.lowerModuleIndices"),
    "t5": ("t5.nQuintuplets", "t5.totOccupancyQuintuplets", "t5.lowerModuleIndices"),
}


def _module_of(store, obj, idx):
    name = _CAP_FIELDS[store][2]
    arr = obj.get(name)
    mult = {"md": 1, "ls": 1, "t3": 3, "t5": 5}[store]
    return int(arr[mult * idx])


def explain_differences(a, b, tr: Tracer, diff: dict | None = None, use_dnn: bool = True) -> list:
    """Every root flip and every T5 flag difference between two sides
    (oracle.identity.Objects a and b of the same event, the event already set
    on the tracer), each with its explanation:

      cut        traced to one comparison decided differently by the two
                 single-precision arithmetics ("explained": its exact margin
                 is within the rounding error of the margin);
      duplicate  a T5 duplicate-removal comparison (trace_t5_state);
      cap shift  the object passes in both arithmetics but its module
                 overflowed its occupancy cap and holds a different number of
                 candidates on the two sides: a flip of another candidate of
                 the same module changed which ones fit under the cap.
    """
    from . import identity

    d = diff if diff is not None else identity.diff(a, b)
    out = []
    for st in ("md", "ls", "t3", "t5", "pt3", "pt5"):
        r = d[st]
        ca = {}
        for side_name, side, other, n_only in (("a", a, b, r["root_only_a"]), ("b", b, a, r["root_only_b"])):
            if not n_only:
                continue
            mine = [k for k in (set(side.keys[st]) - set(other.keys[st]))]
            st_other = other.state_map()
            st_mine = side.state_map()
            pos = {k: j for j, k in enumerate(side.keys[st])}
            for k in mine:
                parts = side.parts[st][pos[k]]
                if not all(pk in st_other[ps] and st_other[ps][pk] == st_mine[ps].get(pk) for ps, pk in parts):
                    continue  # a cascade
                e = tr.trace_flip(st, k, use_dnn)
                e["side"] = side_name
                e["kind"] = "cut"
                if not e["explained"] and e.get("pass_cr") == e.get("pass_glibc") and st in _CAP_FIELDS:
                    mod = _module_of(st, side, int(side.index[st][pos[k]]))
                    nf, tf, _ = _CAP_FIELDS[st]
                    n_a, t_a = int(a.get(nf)[mod]), int(a.get(tf)[mod])
                    n_b, t_b = int(b.get(nf)[mod]), int(b.get(tf)[mod])
                    if (t_a > n_a or t_b > n_b) and t_a != t_b:
                        e.update({"kind": "cap shift", "explained": True, "module": mod,
                                  "occupancy": {"a": [n_a, t_a], "b": [n_b, t_b]}})
                out.append(e)
    # T5 flag differences (duplicate removal)
    allk = set(a.keys["t5"]) | set(b.keys["t5"])
    by_hit = {}
    for k in allk:
        for h in set(k):
            by_hit.setdefault(h, []).append(k)
    sa, sb = a.state_map()["t5"], b.state_map()["t5"]
    for k in set(sa) & set(sb):
        fa, fb = sa[k], sb[k]
        if fa[:2] == fb[:2]:
            continue  # only partOfPT5 differs: a cascade of a pT5 difference
        cand = set()
        for h in set(k):
            cand.update(by_hit.get(h, []))
        partners = [p for p in cand if p != k and shared_hits(p, k) >= 5]
        partners.sort()
        e = trace_t5_state(tr, k, partners, use_dnn)
        e["flags"] = {"a": list(fa), "b": list(fb)}
        if not e["explained"] and fa[1] != fb[1]:
            e["reason"] = "TightCutFlag differs"
        out.append(e)
    return out


# Stored outputs compared with the FP64 re-evaluation, per store, and the
# ones of order one (angles, eta, the DNN score in [0, 1]) that are compared
# with an absolute tolerance below 1.
FP64_FIELDS = {
    "t5": ("innerRadius", "bridgeRadius", "outerRadius", "pt", "eta", "phi", "score_rphisum", "regressionRadius",
           "regressionG", "regressionF", "rzChiSquared", "chiSquared", "nonAnchorChiSquared"),
    "pt3": ("pixelRadius", "tripletRadius", "pt", "eta", "phi", "score", "rPhiChiSquared", "rPhiChiSquaredInwards",
            "rzChiSquared"),
    "pt5": ("pixelRadius", "quintupletRadius", "score", "eta", "phi", "centerX", "centerY", "rzChiSquared",
            "rPhiChiSquared", "rPhiChiSquaredInwards"),
}
ANGLES = {"eta", "phi", "dnnScore"}


def fp64_deviations(obj, tr: Tracer, stores=("t5", "pt3", "pt5"), use_dnn: bool = True) -> dict:
    """For every object of the given stores: its stored floats (obj, an
    oracle.identity.Objects whose event is set on the tracer) against the
    FP64 re-evaluation from its hits.  Returns {"store.field": (stored,
    fp64)} arrays, plus "t5.dnnScore" (the classifier score, which the
    reference does not store: single-precision evaluation with the CUDA
    path's arithmetic against FP64)."""
    out = {}
    for st in stores:
        fields = FP64_FIELDS[st]
        stored = {f: obj.get(f"{st}.{f}") for f in fields}
        s_vals = {f: [] for f in fields}
        f_vals = {f: [] for f in fields}
        dnn32, dnn64 = [], []
        for j, k in enumerate(obj.keys[st]):
            i = int(obj.index[st][j])
            v64 = tr.values(st, k, MODE_F64, use_dnn)
            for f in fields:
                s_vals[f].append(float(stored[f][i]))
                f_vals[f].append(v64[f])
            if st == "t5":
                dnn64.append(v64["dnnScore"])
                dnn32.append(tr.values(st, k, MODE_CR, use_dnn)["dnnScore"])
        for f in fields:
            out[f"{st}.{f}"] = (np.array(s_vals[f]), np.array(f_vals[f]))
        if st == "t5":
            out["t5.dnnScore"] = (np.array(dnn32), np.array(dnn64))
    return out


def deviation_stats(pairs: dict, tol: float = 1e-5) -> dict:
    """Per field: count, fraction within tol (relative; absolute below 1 for
    the fields of ANGLES), median and largest deviation on that scale."""
    res = {}
    for name, (s, f) in pairs.items():
        ok = np.isfinite(s) & np.isfinite(f)
        s, f = s[ok], f[ok]
        field = name.split(".", 1)[1]
        scale = np.maximum(np.abs(f), 1.0) if field in ANGLES else np.abs(f)
        dev = np.abs(s - f)
        rel = np.where(scale > 0, dev / np.where(scale > 0, scale, 1), np.where(dev > 0, np.inf, 0.0))
        res[name] = {"n": int(rel.size), "within": float(np.mean(rel <= tol)) if rel.size else 1.0,
                     "median": float(np.median(rel)) if rel.size else 0.0,
                     "max": float(np.max(rel)) if rel.size else 0.0}
    return res
