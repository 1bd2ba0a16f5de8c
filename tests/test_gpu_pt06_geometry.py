"""PU200-shaped events on the pt0.6 module and pixel maps (OT800_IT615_pt0.6,
pt cut 0.6 GeV in every cut that uses it).  The reference cannot load these
maps (its 40-entry module-map rows hold fewer connections than 1328 modules
list), so no reference run pins the results; checked here instead:

* batched and per-event runs give identical track candidates;
* the tracer (oracle/tracer.py, the same cut code compiled for the host in
  single precision) re-evaluates every stored T5 / pT3 / pT5 and a sample of
  MDs, segments and triplets from their hits on the pt0.6 event setup,
  accepts each and reproduces every stored float bit for bit;
* the looser maps and cut find more segments and triplets than pt0.8."""
import numpy as np
import pytest

from oracle import identity, tracer
from tracklooper_b200 import gen, geometry, lst

pytestmark = pytest.mark.gpu

PT06 = "OT800_IT615_pt0.6"


def test_pt06_events():
    if not tracer.available():
        pytest.fail("oracle/_ref/liblsttrace.so is not built")
    es06 = lst.ES(device=0, geometry_dir=geometry.geometry_dir(PT06))
    es08 = lst.ES(device=0)
    assert es06.info["ptCut"] == pytest.approx(0.6)
    inputs = [gen.generate_event(2, 30 + i) for i in range(2)]
    max_hits = max(i.n_hits for i in inputs) + 1024
    tr = tracer.Tracer(geometry_dir=geometry.geometry_dir(PT06))
    try:
        batch = lst.EventSet(es06, n_slots=2, max_hits=max_hits)
        blob, offsets = lst.pack_events(inputs)
        batch.upload_packed(0, blob, offsets)
        batch.run(0, 2)
        out_b = batch.output(0, 2, tc_capacity=2 * 31000, hits_capacity=2 * 31000 * 14)
        counts06 = batch.batch_counts(0, 2)
        for slot, inp in enumerate(inputs):
            ev = lst.Event(es06, max_hits=max_hits)
            ev.run(inp)
            h1, l1, s1, t1 = ev.getOutput()
            a, b = int(out_b[4][slot]), int(out_b[4][slot + 1])
            assert np.array_equal(out_b[1][a:b], l1) and np.array_equal(out_b[3][a:b], t1)
            # the tracer accepts and reproduces the stored objects
            obj = identity.Objects(ev.field, es06.info["nLowerModules"], inp.n_hits)
            tr.set_event(inp)
            pixel_md = set(int(i) for i in obj.si.md_pixel)
            bad, n = [], 0
            for st, stride in (("md", 97), ("ls", 97), ("t3", 53), ("t5", 1), ("pt3", 1), ("pt5", 1)):
                names = [f for f in tracer.VALUE_NAMES[st] if f not in ("dnnScore", "pixelRadiusError")]
                arrays = {f: ev.field(f"{st}.{f}") for f in names}
                for j in range(0, len(obj.keys[st]), stride):
                    i = int(obj.index[st][j])
                    if st == "md" and i in pixel_md:
                        continue
                    ok, vals, _, _ = tr.eval(st, obj.keys[st][j], tracer.MODE_CR)
                    n += 1
                    if not ok:
                        bad.append((st, obj.keys[st][j], "rejected"))
                    for f in names:
                        if np.float32(vals[f]).view(np.uint32) != np.float32(arrays[f][i]).view(np.uint32):
                            bad.append((st, obj.keys[st][j], f))
            assert n > 3000 and not bad, bad[:5]
            ev.event_set.close()
        batch.close()
        ev08 = lst.Event(es08, max_hits=max_hits)
        ev08.run(inputs[0])
        c08 = ev08.counts()
        ev08.event_set.close()
        assert counts06[0]["nSegments"] > c08["nSegments"] and counts06[0]["nTriplets"] > c08["nTriplets"]
    finally:
        tr.close()
        es06.close()
        es08.close()
