"""Learned boundary-state speculation: the MLP's tensor-core gradients against
a float64 CPU reference, the speculative lexer's tokens against the oracle
(exact for any weights), and what the trained network gains over guessing
one state at every boundary."""

import numpy as np
import pytest

import oracle
from oracle import mlp as mref
from alpacc_b200 import synth, tables

pytestmark = pytest.mark.gpu
_CACHE = {}


def _g(name):
    from alpacc_b200.api import Grammar
    if name not in _CACHE:
        tb = tables.load(name, "lexer")
        _CACHE[name] = (Grammar(tb), oracle.Oracle(tb.blob()))
    return _CACHE[name]


def _doc(name, size, seed):
    return (synth.json_doc(size, 8, seed) if name == "json" else synth.sexp_doc(size, 20, seed)).tobytes()


def test_mlp_gradients_match_float64_reference(has_gpu):
    """Every parameter block's gradient within 2% relative L2 error of the
    float64 restatement (which uses the same BF16 rounding points); the loss
    within 1e-3 relative."""
    import torch
    from alpacc_b200 import spec
    g, _ = _g("json")
    m = spec.BoundaryModel(g, seed=3)
    rng = np.random.default_rng(4)
    M = 64
    win = rng.integers(0, 256, size=(M, 64), dtype=np.uint8)
    lab = rng.integers(0, m.n_states, size=M, dtype=np.uint8)
    loss, _ = m.train_step(torch.from_numpy(win).cuda(), torch.from_numpy(lab).cuda(), update=False)
    got = m.grads.cpu().numpy().astype(np.float64)
    rloss, want, _ = mref.forward_backward(m.params.cpu().numpy(), win, lab, m.n_states)
    assert abs(loss - rloss) <= 1e-3 * abs(rloss)
    blocks = {"emb": (mref.P_EMB, mref.P_W1), "w1": (mref.P_W1, mref.P_B1), "b1": (mref.P_B1, mref.P_W2),
              "w2": (mref.P_W2, mref.P_B2), "b2": (mref.P_B2, mref.P_W3), "w3": (mref.P_W3, mref.P_B3),
              "b3": (mref.P_B3, mref.P_TOTAL)}
    for name, (a, b) in blocks.items():
        err = np.linalg.norm(got[a:b] - want[a:b]) / max(np.linalg.norm(want[a:b]), 1e-30)
        assert err < 2e-2, (name, err)


def _with_mlp_kernel(g, which):
    cfg = g.get_tuning()
    g.set_tuning(cfg[:3] + [which])
    return cfg


def _ref_argmax(m, d, pos):
    x = np.frombuffer(d, np.uint8)
    idx = pos[:, None] - 64 + np.arange(64)[None, :]
    win = np.where((idx >= 0) & (idx < len(x)), x[np.clip(idx, 0, len(x) - 1)], 0x20).astype(np.uint8)
    _, _, logits = mref.forward_backward(m.params.cpu().numpy(), win, np.zeros(len(pos), np.int64), m.n_states)
    return logits.argmax(axis=1)


@pytest.mark.parametrize("kernel", [0, 1], ids=["tcgen05", "mma_sync"])
def test_mlp_predict_matches_reference(has_gpu, kernel):
    """Each inference kernel's argmax against the float64 forward pass
    (>= 99% agreement: rows whose top two logits are closer than the
    FP32/BF16 rounding may differ)."""
    from alpacc_b200 import spec
    g, _ = _g("json")
    saved = _with_mlp_kernel(g, kernel)
    try:
        m = spec.BoundaryModel(g, seed=5)
        d = _doc("json", 200000, 21)
        pos = np.arange(1, 1000) * 160
        pred = m.predict(d, pos).cpu().numpy()
        assert np.mean(pred == _ref_argmax(m, d, pos)) >= 0.99
    finally:
        g.set_tuning(saved)


def test_mlp_tcgen05_kernel_agrees_with_mma_sync(has_gpu):
    """The tcgen05 kernel (tensor-memory accumulators, swizzled shared-memory
    operands) against the mma.sync kernel: same rounding points, different
    summation order, so the argmax agrees except on near ties.  Ragged tile
    counts, windows reaching before the input's start and past its end, and
    more tiles than SMs (several tiles per CTA, the stage ring wrapping)."""
    from alpacc_b200 import spec
    g, _ = _g("json")
    saved = g.get_tuning()
    try:
        m = spec.BoundaryModel(g, seed=7)
        d = _doc("json", 3 << 20, 23)
        rng = np.random.default_rng(8)
        for count in (1, 127, 128, 129, 1000, 19000, 60000):
            pos = np.sort(rng.integers(0, len(d) + 100, count))
            pos[:min(count, 3)] = [0, 5, 63][:min(count, 3)]
            got = {}
            for k in (0, 1):
                g.set_tuning(saved[:3] + [k])
                got[k] = m.predict(d, pos).cpu().numpy()
            assert got[0].max() < m.n_states
            assert np.mean(got[0] == got[1]) >= 0.995, count
            if count <= 1000:
                assert np.mean(got[0] == _ref_argmax(m, d, pos)) >= 0.99, count
    finally:
        g.set_tuning(saved)


@pytest.mark.parametrize("name", ["json", "sexp"])
@pytest.mark.parametrize("chunk", [128, 256, 1024, 4096])
def test_speculative_tokens_exact(has_gpu, name, chunk):
    from alpacc_b200 import spec
    g, o = _g(name)
    for kind, m in (("random", spec.BoundaryModel(g, seed=1)), ("constant", spec.BoundaryModel.constant(g, 1))):
        for i, size in enumerate([1, 100, chunk, chunk + 1, 3 * chunk + 17, 300_000]):
            d = _doc(name, size, 900 + i)
            want = o.lex_futhark(d)
            got, stats = m.lex(d, chunk)
            if want is None:
                assert got is None
                continue
            assert got is not None, (kind, size)
            for a, b in zip(got, want):
                np.testing.assert_array_equal(a.cpu().numpy().astype(b.dtype), b)
        bad = b'{"a": [1, 2, "x' + b" " * 5000
        assert m.lex(bad, chunk)[0] is None


def test_trained_network_beats_constant_guess(has_gpu):
    """Train on labelled boundaries of distinct documents, then compare the
    hit rate at unseen chunk boundaries with guessing the most frequent state."""
    import torch
    from alpacc_b200 import spec
    g, o = _g("json")
    train_docs = [synth.json_doc(1 << 20, 8, 0xA1FACC10 + k) for k in range(8)]
    win, lab = spec.dataset(g, train_docs, per_doc=40000, seed=7)
    m = spec.BoundaryModel(g, seed=0)
    info = m.train(win, lab, epochs=3, batch=4096, lr=3e-3)
    freq = int(torch.bincount(lab.long()).argmax())
    const = spec.BoundaryModel.constant(g, freq)
    test = synth.json_doc(4 << 20, 8, 0xA1FACC20)
    st = spec.exact_states(g, test)
    C = 1024
    pos = np.arange(1, len(test) // C) * C
    truth = st[torch.as_tensor(pos // 16)].cpu().numpy()
    hit_m = float(np.mean(m.predict(test, pos).cpu().numpy() == truth))
    hit_c = float(np.mean(const.predict(test, pos).cpu().numpy() == truth))
    _, s_m = m.lex(test, C)
    _, s_c = const.lex(test, C)
    print("trained hit %.4f (mismatch %d, reruns %d) vs constant %.4f (mismatch %d, reruns %d); %s"
          % (hit_m, s_m[1], s_m[2], hit_c, s_c[1], s_c[2], info))
    assert hit_m > hit_c + 0.05
    assert s_m[2] < s_c[2]
