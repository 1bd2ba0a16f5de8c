"""Training the T5 classifier on the pipeline's own quintuplet candidates.

The classifier is the reference's 38 -> 32 (ReLU) -> 32 (ReLU) -> 1 (sigmoid)
MLP (SDL/NeuralNetwork.h).  Training data are the quintuplet candidates that
pass every cut before the DNN decision, dumped by the CUDA probe
(lst_batch_t5_probe) from seeded synthetic events; labels come from the
generator's sim-hit truth with the reference's rule (code/core/trkCore.cc:
231-403: a candidate is true when more than 75% of its distinct hits come
from one simulated particle).

The network's forward and backward passes are this project's CUDA kernels
(lst_t5dnn_forward / lst_t5dnn_backward) behind ``T5DnnFunction``, a
torch.autograd.Function; torch only supplies the loss, Adam and the tensors.

  python -m tracklooper_b200.t5dnn --train-events 2000 --test-events 256 \
      --out t5dnn_retrained.bin
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import gen, lst

N_PARAMS = 2337
N_FEATURES = 38
REFERENCE_WP = 0.6177366
# parameter offsets in the weight-file layout
W0, B0, W2, B2, W4, B4 = 0, 1216, 1248, 2272, 2304, 2336


def _torch():
    import torch

    return torch


def _check_dnn(rc, what):
    if rc < 0:
        raise lst.LSTError(f"{what}: {lst.library().lst_t5dnn_last_error().decode(errors='replace')}")


def _make_function():
    torch = _torch()

    class T5DnnFunction(torch.autograd.Function):
        """logits = MLP(x; weights) with the project's CUDA forward/backward."""

        @staticmethod
        def forward(ctx, x, weights):
            lib = lst.library()
            x = x.contiguous()
            weights = weights.contiguous()
            n = x.shape[0]
            h1 = torch.empty(n, 32, device=x.device, dtype=torch.float32)
            h2 = torch.empty(n, 32, device=x.device, dtype=torch.float32)
            logit = torch.empty(n, device=x.device, dtype=torch.float32)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            _check_dnn(lib.lst_t5dnn_forward(weights.data_ptr(), x.data_ptr(), n, h1.data_ptr(), h2.data_ptr(),
                                             logit.data_ptr(), stream), "lst_t5dnn_forward")
            ctx.save_for_backward(x, weights, h1, h2)
            return logit

        @staticmethod
        def backward(ctx, dlogit):
            lib = lst.library()
            x, weights, h1, h2 = ctx.saved_tensors
            n = x.shape[0]
            dlogit = dlogit.contiguous().to(torch.float32)
            grad = torch.empty(N_PARAMS, device=x.device, dtype=torch.float32)
            scratch = torch.empty(int(lib.lst_t5dnn_scratch_floats(n)), device=x.device, dtype=torch.float32)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            _check_dnn(lib.lst_t5dnn_backward(weights.data_ptr(), x.data_ptr(), h1.data_ptr(), h2.data_ptr(),
                                              dlogit.data_ptr(), n, grad.data_ptr(), scratch.data_ptr(), stream),
                       "lst_t5dnn_backward")
            return None, grad

    return T5DnnFunction


_FN = None


def t5dnn_logits(x, weights):
    """Logits of the T5 DNN for features x (n x 38, CUDA float32)."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN.apply(x, weights)


def torch_reference_logits(x, weights):
    """The same network written with torch operations (for checking)."""
    torch = _torch()
    w0 = weights[W0:B0].reshape(38, 32)
    h1 = torch.relu(x @ w0 + weights[B0:W2])
    h2 = torch.relu(h1 @ weights[W2:B2].reshape(32, 32) + weights[B2:W4])
    return h2 @ weights[W4:B4] + weights[B4]


def numpy_logits(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """float64 restatement on the host (finite-difference checks)."""
    x = x.astype(np.float64)
    w = w.astype(np.float64)
    h1 = np.maximum(x @ w[W0:B0].reshape(38, 32) + w[B0:W2], 0.0)
    h2 = np.maximum(h1 @ w[W2:B2].reshape(32, 32) + w[B2:W4], 0.0)
    return h2 @ w[W4:B4] + w[B4]


def reference_weights() -> np.ndarray:
    return np.fromfile(lst.DNN_WEIGHTS, dtype="<f4")


RETRAINED_WEIGHTS = lst.DNN_WEIGHTS.replace("t5dnn_reference.bin", "t5dnn_retrained.bin")


def retrained_weights() -> tuple[np.ndarray, float]:
    """The committed retrained weights and their working point."""
    with open(RETRAINED_WEIGHTS.replace(".bin", ".json")) as f:
        wp = float(json.load(f)["working_point"])
    return np.fromfile(RETRAINED_WEIGHTS, dtype="<f4"), wp


def random_weights(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases."""
    rng = np.random.default_rng(seed)
    w = np.zeros(N_PARAMS, np.float32)
    w[W0:B0] = rng.normal(0, np.sqrt(2.0 / 38), 38 * 32)
    w[W2:B2] = rng.normal(0, np.sqrt(2.0 / 32), 32 * 32)
    w[W4:B4] = rng.normal(0, np.sqrt(1.0 / 32), 32)
    return w


# ------------------------------------------------------------------ truth
def truth_labels(hits: np.ndarray, hit_sim: np.ndarray) -> np.ndarray:
    """1 where more than 75% of a candidate's distinct hits come from one
    simulated particle (code/core/trkCore.cc:231-403; one sim particle per
    hit here, -1 for noise).  hits: (n, k) event-local hit indices."""
    hits = np.asarray(hits, np.int64)
    if hits.shape[0] == 0:
        return np.zeros(0, np.int8)
    h = np.sort(hits, axis=1)
    uniq = np.ones_like(h, dtype=bool)
    uniq[:, 1:] = h[:, 1:] != h[:, :-1]
    sims = np.asarray(hit_sim, np.int64)[h]
    n_uniq = uniq.sum(axis=1)
    # for each distinct hit, how many distinct hits share its particle
    same = (sims[:, :, None] == sims[:, None, :]) & uniq[:, None, :]
    counts = np.where(uniq, same.sum(axis=2), 0)
    best = counts.argmax(axis=1)
    best_sim = sims[np.arange(h.shape[0]), best]
    best_cnt = counts[np.arange(h.shape[0]), best]
    return ((best_sim >= 0) & (best_cnt > 0.75 * n_uniq)).astype(np.int8)


# ------------------------------------------------------------ candidates
def collect_candidates(es: lst.ES, inputs, batch: int = 32, capacity: int = 1 << 21, eset: lst.EventSet = None):
    """Runs the chain up to the quintuplet stage on `inputs` and returns the
    classifier-stage candidates: dict of features, loaded weights' score,
    cut-only decision, rz tight flag, truth label and event index.  Uses
    `eset` if given (its hit capacity must hold the inputs)."""
    torch = _torch()
    lib = lst.library()
    dev = torch.device("cuda", es.device)
    own = eset is None
    if own:
        max_hits = max(i.n_hits for i in inputs) + 1024
        eset = lst.EventSet(es, n_slots=min(batch, len(inputs)), max_hits=max_hits)
    feat = torch.empty(capacity, 38, device=dev)
    score = torch.empty(capacity, device=dev)
    cut = torch.empty(capacity, dtype=torch.uint8, device=dev)
    tight = torch.empty(capacity, dtype=torch.uint8, device=dev)
    hits = torch.empty(capacity, 10, dtype=torch.int32, device=dev)
    evi = torch.empty(capacity, dtype=torch.int32, device=dev)
    parts = []
    for b0 in range(0, len(inputs), eset.n_slots):
        chunk = inputs[b0:b0 + eset.n_slots]
        blob, off = lst.pack_events(chunk)
        eset.upload_packed(0, blob, off)
        eset.run(0, len(chunk), lst.STAGE_MINI_DOUBLETS, lst.STAGE_QUINTUPLETS)
        n = ctypes.c_uint32()
        lst._check(lib.lst_batch_t5_probe(eset.handle, 0, len(chunk), feat.data_ptr(), score.data_ptr(),
                                          cut.data_ptr(), tight.data_ptr(), hits.data_ptr(), evi.data_ptr(),
                                          capacity, ctypes.byref(n)), "lst_batch_t5_probe")
        k = min(n.value, capacity)
        if n.value > capacity:
            raise RuntimeError(f"probe capacity {capacity} exceeded ({n.value})")
        h = hits[:k].cpu().numpy().view(np.uint32)
        e = evi[:k].cpu().numpy()
        lab = np.zeros(k, np.int8)
        for j in np.unique(e):
            sel = e == j
            lab[sel] = truth_labels(h[sel], chunk[j].hit_sim)
        parts.append({"feat": feat[:k].cpu().numpy().copy(), "score": score[:k].cpu().numpy().copy(),
                      "cut": cut[:k].cpu().numpy().copy(), "tight": tight[:k].cpu().numpy().copy(),
                      "label": lab, "event": e + b0})
    if own:
        eset.close()
    data = {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}
    # the probe appends in no fixed order: sort by (event, features) so that the
    # data set, and with it training, is reproducible
    keys = [data["feat"][:, k] for k in range(37, -1, -1)] + [data["event"]]
    order = np.lexsort(keys)
    return {k: v[order] for k, v in data.items()}


def generate(config: int, first: int, n: int, workers: int = 16):
    with ThreadPoolExecutor(max_workers=workers) as pool:
        return list(pool.map(lambda i: gen.generate_event(config, first + i), range(n)))


# -------------------------------------------------------------- training
def fold_standardisation(w: np.ndarray, mean: np.ndarray, std: np.ndarray) -> np.ndarray:
    """Weights acting on raw features, from weights trained on (x - mean) / std."""
    out = w.astype(np.float64).copy()
    w0 = out[W0:B0].reshape(38, 32)
    b0 = out[B0:W2]
    b0 -= (mean / std) @ w0
    w0 /= std[:, None]
    out[W0:B0] = w0.ravel()
    out[B0:W2] = b0
    return out.astype(np.float32)


def train(data: dict, epochs: int = 30, batch: int = 8192, lr: float = 1e-3, seed: int = 0, device: int = 0,
          log=None) -> tuple[np.ndarray, list]:
    """Adam on binary cross-entropy, FP32, the project's forward/backward
    kernels.  Inputs are standardised for training and the standardisation is
    folded into the first layer of the returned weights."""
    torch = _torch()
    dev = torch.device("cuda", device)
    x = data["feat"].astype(np.float32)
    y = data["label"].astype(np.float32)
    mean = x.mean(axis=0).astype(np.float64)
    std = x.std(axis=0).astype(np.float64)
    std[std < 1e-6] = 1.0
    xs = torch.tensor(((x - mean) / std).astype(np.float32), device=dev)
    yt = torch.tensor(y, device=dev)
    w = torch.tensor(random_weights(seed), device=dev, requires_grad=True)
    opt = torch.optim.Adam([w], lr=lr)
    gen_ = torch.Generator(device="cpu").manual_seed(seed)
    n = xs.shape[0]
    history = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen_).to(dev)
        tot = 0.0
        t0 = time.perf_counter()
        for b in range(0, n, batch):
            idx = perm[b:b + batch]
            logit = t5dnn_logits(xs[idx], w)
            loss = torch.nn.functional.binary_cross_entropy_with_logits(logit, yt[idx])
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            tot += float(loss) * idx.numel()
        history.append({"epoch": ep, "loss": tot / n, "seconds": time.perf_counter() - t0})
        if log:
            log(f"epoch {ep}: loss {tot / n:.5f}")
    return fold_standardisation(w.detach().cpu().numpy(), mean, std), history


def scores(data: dict, w: np.ndarray, device: int = 0) -> np.ndarray:
    torch = _torch()
    dev = torch.device("cuda", device)
    with torch.no_grad():
        x = torch.tensor(data["feat"].astype(np.float32), device=dev)
        logit = t5dnn_logits(x, torch.tensor(w, device=dev))
        return torch.sigmoid(logit).cpu().numpy()


def metrics(passed: np.ndarray, label: np.ndarray) -> dict:
    """Candidate-level efficiency (passing true / all true) and fake rate
    (passing fake / all passing)."""
    passed = passed.astype(bool)
    true = label.astype(bool)
    n_true = int(true.sum())
    n_pass = int(passed.sum())
    return {"efficiency": (int((passed & true).sum()) / n_true) if n_true else 0.0,
            "fake_rate": (int((passed & ~true).sum()) / n_pass) if n_pass else 0.0,
            "passed": n_pass, "true": n_true}


def threshold_for_efficiency(score: np.ndarray, label: np.ndarray, efficiency: float) -> float:
    """The working point at which the true-candidate efficiency equals `efficiency`."""
    s = np.sort(score[label.astype(bool)])
    if s.size == 0:
        return 0.5
    k = int(np.floor((1.0 - efficiency) * s.size))
    k = min(max(k, 0), s.size - 1)
    return float(np.nextafter(np.float32(s[k]), np.float32(-1))) if k > 0 else float(s[0]) - 1e-7


def compare(data: dict, w: np.ndarray, wp: float, device: int = 0) -> dict:
    """Reference-weight DNN vs retrained DNN (at working point wp) vs cut-only."""
    lab = data["label"]
    ours = scores(data, w, device)
    return {"reference_dnn": metrics(data["score"] > REFERENCE_WP, lab),
            "retrained_dnn": metrics(ours > wp, lab),
            "cut_only": metrics(data["cut"] != 0, lab)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-events", type=int, default=2000)
    ap.add_argument("--test-events", type=int, default=256)
    ap.add_argument("--test-config", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--out", default="t5dnn_retrained.bin")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    es = lst.ES(device=args.device)
    t0 = time.perf_counter()
    train_data = collect_candidates(es, generate(2, 100000, args.train_events))
    test_data = collect_candidates(es, generate(args.test_config, 200000, args.test_events))
    t1 = time.perf_counter()
    w, hist = train(train_data, epochs=args.epochs, device=args.device, log=print)
    t2 = time.perf_counter()
    # match the reference DNN's efficiency on the training candidates
    ref_eff = metrics(train_data["score"] > REFERENCE_WP, train_data["label"])["efficiency"]
    wp = threshold_for_efficiency(scores(train_data, w, args.device), train_data["label"], ref_eff)
    w.astype("<f4").tofile(args.out)
    res = {"train_candidates": int(train_data["label"].size), "train_true": int(train_data["label"].sum()),
           "test_candidates": int(test_data["label"].size), "working_point": wp,
           "collect_seconds": t1 - t0, "train_seconds": t2 - t1, "final_loss": hist[-1]["loss"],
           "train": compare(train_data, w, wp, args.device), "test": compare(test_data, w, wp, args.device)}
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
