"""pLS duplicate removal on pLS that share pixel hits, against the reference
CPU backend.

The generated events give every pLS hits of its own, so their cleaning passes
remove pLS only through the second pass's dR2 test.  Here a pileup event gets
extra pLS copied from its own with one to four hits in common with the
original (in its order or permuted), with the kinematics kept, nudged or moved
beyond the 0.1 eta window, and with some quads turned into triplets; in one
case some copies and some originals get a NaN or infinite eta.  The full list
is then shuffled, so that the copy is sometimes the lower index and
sometimes the higher.  Every store must match the reference's after each
stage, and both passes must have marked pLS.
"""
import dataclasses

import numpy as np
import pytest

from oracle import compare, reflib
from tracklooper_b200 import gen, lst

pytestmark = pytest.mark.gpu

STAGES = ("md", "ls", "t3", "t5", "pls_clean", "pt5", "pt3", "tc")


def _with_shared_hit_pls(inp, n_extra, seed, n_nonfinite=0):
    rng = np.random.default_rng(seed)
    p = {k: np.asarray(v) for k, v in inp.pls.items()}
    n = inp.n_pls
    hits = np.stack([p[f"hitIndices{i}"] for i in range(4)], 1)
    extra = {k: [] for k in p}
    extra_sim = []
    for m, j in enumerate(rng.choice(n, n_extra, replace=False)):
        row = {k: v[j].copy() for k, v in p.items()}
        h = hits[j].copy()
        other = hits[rng.integers(n)]
        kind = m % 7
        if kind == 1:  # three in common
            h[3] = other[3]
        elif kind == 2:  # two in common
            h[1:3] = other[1:3]
        elif kind == 3:  # one in common
            h[1:] = other[1:]
        elif kind == 4:  # all four, permuted
            h = h[[2, 0, 3, 1]]
        elif kind == 5:  # none in common, at dR below 1e-5 of the original
            h = other.copy()
        elif kind == 6:  # three in common, as a triplet
            h[3] = h[2]
            row["isQuad"] = np.int8(0)
        if kind in (1, 2, 3, 4) and m % 3 == 0:
            row["eta"] = np.float32(row["eta"] + rng.choice([0.03, -0.06, 0.12, -0.2]))
        if kind == 5:
            row["eta"] = np.float32(row["eta"] + 1e-3)
            row["phi"] = np.float32(row["phi"] - 1e-3)
        if m % 5 == 0:
            row["ptErr"] = np.float32(row["ptErr"] * 1.5)
        for i in range(4):
            row[f"hitIndices{i}"] = h[i]
        for k in p:
            extra[k].append(row[k])
        extra_sim.append(inp.pls_sim[j])
    order = rng.permutation(n + n_extra)
    pls = {k: np.concatenate([p[k], np.array(extra[k], dtype=p[k].dtype)])[order] for k in p}
    pls_sim = np.concatenate([inp.pls_sim, np.array(extra_sim, dtype=inp.pls_sim.dtype)])[order]
    if n_nonfinite:
        # NaN and infinite eta on copies (which share hits with others) and on
        # originals: a NaN never satisfies the reference's |deta| > 0.1 skip
        copies = rng.choice(np.nonzero(order >= n)[0], n_nonfinite, replace=False)
        originals = rng.choice(np.nonzero(order < n)[0], n_nonfinite, replace=False)
        for k, i in enumerate(np.concatenate([copies, originals])):
            pls["eta"][i] = (np.nan, np.inf, -np.inf)[k % 3]
    return dataclasses.replace(inp, pls=pls, pls_sim=pls_sim, seeds=None)


@pytest.fixture(scope="module")
def ref():
    if not reflib.available("cr"):
        pytest.fail("reference library oracle/_ref/liblstref_cr.so is not built")
    r = reflib.RefLST("cr")
    yield r
    r.close()


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


@pytest.mark.parametrize("config,index,n_extra,n_nonfinite", [(2, 5, 700, 0), (3, 2, 300, 0), (3, 4, 300, 24)])
def test_shared_hit_pls_match_reference(ref, es, config, index, n_extra, n_nonfinite):
    inp = _with_shared_hit_pls(gen.generate_event(config, index), n_extra, seed=17 + index, n_nonfinite=n_nonfinite)
    ev = lst.Event(es, max_hits=inp.n_hits + 1024)
    dtypes = lst.field_dtypes()
    names = list(dtypes)
    sizes = {"H": ev.event_set.max_hits, "MD": es.info["nTotalMDs"], "LS": es.info["nTotalSegments"],
             "T3": es.info["maxTriplets"], "T5": es.info["maxQuintuplets"]}
    ref.reset()
    ref.add_inputs(inp)
    ev.event_set.add_inputs(0, inp)
    problems = []
    try:
        for st in STAGES:
            ref.run_stage(st)
            ev.event_set.run_stage(0, st)
            p = compare.compare_stores(lambda n: ev.field(n), lambda n: ref.field(n, dtype=dtypes[n]),
                                       compare.stage_fields(names, [st]), es.info["nLowerModules"], inp.n_hits, sizes)
            if p:
                problems.append(f"[{st}] " + "; ".join(p[:6]))
        is_dup = ev.field("ls.isDup")[: inp.n_pls]
    finally:
        ev.event_set.close()
    assert not problems, "\n".join(problems)
    # both passes removed pLS
    assert np.count_nonzero(is_dup & 1) > 0 and np.count_nonzero(is_dup & 2) > 0
