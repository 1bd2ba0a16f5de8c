"""The T5 classifier's training kernels and the classifier-stage probe."""
import numpy as np
import pytest

from tracklooper_b200 import gen, lst, t5dnn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t

    return t


@pytest.fixture(scope="module")
def es():
    e = lst.ES(device=0)
    yield e
    e.close()


def _inputs(torch, n=1000, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1.5, (n, 38)).astype(np.float32)
    return torch.tensor(x, device="cuda"), x


def test_forward_matches_torch_and_float64(torch):
    w = t5dnn.reference_weights()
    xt, x = _inputs(torch)
    wt = torch.tensor(w, device="cuda")
    ours = t5dnn.t5dnn_logits(xt, wt).cpu().numpy()
    ref32 = t5dnn.torch_reference_logits(xt, wt).cpu().numpy()
    ref64 = t5dnn.numpy_logits(x, w)
    assert np.allclose(ours, ref32, rtol=1e-5, atol=1e-5)
    assert np.allclose(ours, ref64, rtol=1e-4, atol=1e-4)


def test_backward_matches_autograd(torch):
    xt, _ = _inputs(torch, n=3000, seed=2)
    y = torch.tensor((np.random.default_rng(3).random(3000) > 0.7).astype(np.float32), device="cuda")
    w0 = torch.tensor(t5dnn.random_weights(4), device="cuda")
    w1 = w0.clone().requires_grad_(True)
    torch.nn.functional.binary_cross_entropy_with_logits(t5dnn.t5dnn_logits(xt, w1), y).backward()
    w2 = w0.clone().requires_grad_(True)
    torch.nn.functional.binary_cross_entropy_with_logits(t5dnn.torch_reference_logits(xt, w2), y).backward()
    g1, g2 = w1.grad.cpu().numpy(), w2.grad.cpu().numpy()
    assert np.max(np.abs(g1 - g2)) <= 1e-4 * max(1.0, np.max(np.abs(g2)))


def test_backward_matches_finite_differences(torch):
    xt, x = _inputs(torch, n=200, seed=5)
    y = (np.random.default_rng(6).random(200) > 0.5).astype(np.float64)
    w = t5dnn.random_weights(7)
    wt = torch.tensor(w, device="cuda", requires_grad=True)
    logit = t5dnn.t5dnn_logits(xt, wt)
    torch.nn.functional.binary_cross_entropy_with_logits(logit, torch.tensor(y, device="cuda", dtype=torch.float32)).backward()
    g = wt.grad.cpu().numpy().astype(np.float64)

    def loss(wv):
        z = t5dnn.numpy_logits(x, wv)
        return np.mean(np.logaddexp(0, z) - y * z)

    rng = np.random.default_rng(8)
    idx = np.concatenate([rng.choice(1216, 20, replace=False), 1216 + rng.choice(32, 5, replace=False),
                          1248 + rng.choice(1024, 20, replace=False), 2272 + rng.choice(32, 5, replace=False),
                          2304 + rng.choice(32, 5, replace=False), [2336]])
    w64 = w.astype(np.float64)
    # central differences in float64 with a step small enough not to cross
    # the ReLU kinks of these inputs
    eps = 1e-6
    for i in idx:
        wp_, wm_ = w64.copy(), w64.copy()
        wp_[i] += eps
        wm_[i] -= eps
        fd = (loss(wp_) - loss(wm_)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-3 * max(abs(fd), 1e-3), (i, fd, g[i])


def test_backward_is_deterministic(torch):
    xt, _ = _inputs(torch, n=5000, seed=9)
    w = torch.tensor(t5dnn.random_weights(10), device="cuda", requires_grad=True)
    grads = []
    for _ in range(2):
        w.grad = None
        t5dnn.t5dnn_logits(xt, w).sum().backward()
        grads.append(w.grad.clone())
    assert torch.equal(grads[0], grads[1])


@pytest.fixture(scope="module")
def probe_event(es):
    inp = gen.generate_event(2, 21)
    data = t5dnn.collect_candidates(es, [inp], batch=1)
    return inp, data


def test_probe_counts_match_selected_quintuplets(es, probe_event):
    inp, data = probe_event
    ev = lst.Event(es, max_hits=inp.n_hits + 1024)
    ev.run(inp, upto="t5")
    n_dnn = int(ev.field("t5.totOccupancyQuintuplets").sum())
    ev.event_set.set_t5_method(lst.T5_CUTS)
    ev.run(inp, upto="t5")
    n_cut = int(ev.field("t5.totOccupancyQuintuplets").sum())
    ev.event_set.close()
    assert n_dnn == int((data["score"] > np.float32(t5dnn.REFERENCE_WP)).sum())
    assert n_cut == int((data["cut"] != 0).sum())
    assert data["label"].sum() > 0 and (data["label"] == 0).sum() > 0


def test_training_reduces_loss_and_beats_cut_only(es):
    train = t5dnn.collect_candidates(es, t5dnn.generate(2, 5000, 128))
    test = t5dnn.collect_candidates(es, t5dnn.generate(2, 6000, 32))
    w, hist = t5dnn.train(train, epochs=30, batch=8192)
    assert hist[-1]["loss"] < hist[0]["loss"]
    cut_eff = t5dnn.metrics(train["cut"] != 0, train["label"])["efficiency"]
    wp = t5dnn.threshold_for_efficiency(t5dnn.scores(train, w), train["label"], cut_eff)
    res = t5dnn.compare(test, w, wp)
    # at the cut-only method's efficiency, the trained network keeps fewer fakes
    assert res["retrained_dnn"]["fake_rate"] < res["cut_only"]["fake_rate"]
