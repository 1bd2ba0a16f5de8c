"""The cut-flip tracer and the FP64 re-evaluation oracle, on the CPU.

The tracer (oracle/trace/lst_trace.cc) evaluates single objects again from
their hits with the product's cut code in three arithmetics.  Before its
explanations and FP64 values count for anything it must reproduce the two
single-precision builds exactly: every stored float of every object of the
parity oracle (correctly rounded transcendentals, the CUDA path's
arithmetic) in MODE_CR, and of the stock reference build (glibc float
math) in MODE_GLIBC.  Then:

* every object that one build keeps and the other does not, and every T5
  whose duplicate flag differs, is traced to a comparison decided
  differently by the two arithmetics, whose exact margin is within the
  single-precision rounding error of the margin -- or to an occupancy cap
  whose module holds a different number of candidates;
* the stored outputs (pt, eta, phi, radii, chi-squared values, scores,
  the DNN score) are compared with their FP64 re-evaluation.
"""
import numpy as np
import pytest

from oracle import identity, reflib, tracer
from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.skipif(not (reflib.available("cr") and reflib.available("native") and tracer.available()),
                                 reason="reference builds or tracer not built")


@pytest.fixture(scope="module")
def sides():
    dt = lst.field_dtypes()
    cr, nat = reflib.RefLST("cr"), reflib.RefLST("native")
    tr = tracer.Tracer()
    events = []
    for cfg, idx in ((2, 0), (5, 0)):
        inp = gen.generate_event(cfg, idx)
        cr.run_event(inp)
        nat.run_event(inp)
        a = identity.Objects(lambda f: cr.field(f, dtype=dt[f]), cr.n_lower, inp.n_hits)
        b = identity.Objects(lambda f: nat.field(f, dtype=dt[f]), nat.n_lower, inp.n_hits)
        events.append((inp, a, b))
        # the stores stay readable through a and b only while the next event
        # has not run: keep the arrays each side needs
        for o in (a, b):
            cache = {}
            get = o.get
            o.get = (lambda g, c: (lambda n: c.setdefault(n, g(n))))(get, cache)
            for st in ("t5", "pt3", "pt5"):
                for f in tracer.FP64_FIELDS[st]:
                    o.get(f"{st}.{f}")
            for st, names in tracer.VALUE_NAMES.items():
                for f in names:
                    if f"{st}.{f}" in dt:
                        o.get(f"{st}.{f}")
            for f in ("md.moduleIndices", "md.nMDs", "md.totOccupancyMDs", "ls.innerLowerModuleIndices",
                      "ls.nSegments", "ls.totOccupancySegments", "t3.lowerModuleIndices", "t3.nTriplets",
                      "t3.totOccupancyTriplets", "t5.lowerModuleIndices", "t5.nQuintuplets",
                      "t5.totOccupancyQuintuplets"):
                o.get(f)
    yield tr, events
    tr.close()
    cr.close()
    nat.close()


def _check_reproduces(tr, obj, mode, stores, stride):
    """Evaluates every stride-th object of each store in `mode` and lists the
    stored floats the tracer does not reproduce bit for bit."""
    bad = []
    n = 0
    for st in stores:
        names = [f for f in tracer.VALUE_NAMES[st] if f not in ("dnnScore", "pixelRadiusError")]
        arrays = {f: obj.get(f"{st}.{f}") for f in names}
        for j in range(0, len(obj.keys[st]), stride):
            i = int(obj.index[st][j])
            key = obj.keys[st][j]
            ok, vals, _, _ = tr.eval(st, key, mode)
            for f in names:
                n += 1
                if np.float32(vals[f]).view(np.uint32) != np.float32(arrays[f][i]).view(np.uint32):
                    bad.append((st, key, f, float(arrays[f][i]), vals[f]))
            if not ok:
                bad.append((st, key, "rejected", None, None))
    return n, bad


def test_tracer_reproduces_both_single_precision_builds(sides):
    tr, events = sides
    inp, a, b = events[0]
    tr.set_event(inp)
    pixel_md = set(int(i) for i in a.si.md_pixel)
    # pixel mini-doublets are inputs: leave them out of the MD check
    for o in (a, b):
        keep = [j for j, i in enumerate(o.index["md"]) if int(i) not in pixel_md]
        o.keys["md"] = [o.keys["md"][j] for j in keep]
        o.index["md"] = o.index["md"][keep]
    n1, bad1 = _check_reproduces(tr, a, tracer.MODE_CR, ("md", "ls", "t3", "t5", "pt3", "pt5"), 7)
    n2, bad2 = _check_reproduces(tr, b, tracer.MODE_GLIBC, ("md", "ls", "t3", "t5", "pt3", "pt5"), 7)
    assert n1 > 20000 and n2 > 20000
    assert not bad1, bad1[:5]
    assert not bad2, bad2[:5]


def test_every_difference_is_a_rounding_level_flip(sides):
    tr, events = sides
    total = 0
    for inp, a, b in events:
        tr.set_event(inp)
        d = identity.diff(a, b)
        ex = tracer.explain_differences(a, b, tr, d)
        total += len(ex)
        unexplained = [e for e in ex if not e["explained"]]
        assert not unexplained, unexplained[:3]
        # every root flip of the diff is among the explained ones
        n_root = sum(d[st]["root_only_a"] + d[st]["root_only_b"] for st in ("md", "ls", "t3", "t5", "pt3", "pt5"))
        assert sum(1 for e in ex if e.get("kind") in ("cut", "cap shift")) == n_root
    assert total > 0  # the two builds do differ on these events


def test_fp64_reevaluation_of_stored_outputs(sides):
    """The stored outputs of the CUDA path's arithmetic against FP64.  The
    well-conditioned ones (pt, eta, phi, circle radii, the DNN score) are
    within 1e-5 on at least 98% of the objects.  The chi-squared values and
    the scores built from them are differences of nearly equal sums: their
    single-precision evaluation -- the reference's own formula -- is not
    within 1e-5 of FP64 on most objects, and the stock build is no closer:
    the two builds' median deviations agree within 25%."""
    tr, events = sides
    inp, a, b = events[0]
    tr.set_event(inp)
    sa = tracer.deviation_stats(tracer.fp64_deviations(a, tr))
    sb = tracer.deviation_stats(tracer.fp64_deviations(b, tr))
    well = ("t5.pt", "t5.eta", "t5.phi", "t5.innerRadius", "t5.bridgeRadius", "t5.outerRadius", "t5.dnnScore",
            "pt3.pixelRadius", "pt3.tripletRadius", "pt3.pt", "pt3.eta", "pt3.phi", "pt5.pixelRadius", "pt5.eta",
            "pt5.phi")
    for name in well:
        assert sa[name]["within"] >= 0.98, (name, sa[name])
        assert sa[name]["max"] <= 1e-4, (name, sa[name])
    for name in sa:
        if name in sb and sb[name]["median"] > 0:
            assert 0.8 <= sa[name]["median"] / sb[name]["median"] <= 1.25, (name, sa[name], sb[name])
