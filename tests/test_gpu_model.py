"""The learned warm start's MLP on the tensor cores (tcgen05): inference and gradients against a
numpy f32 reference with the same bf16 roundings, and training that lowers the loss."""
import numpy as np
import pytest

import mlp_reference as ref
from conftest import rp

pytestmark = pytest.mark.gpu


def _data(n, seed):
    r = np.random.default_rng(seed)
    f = r.normal(0.0, 1.0, (n, 24)).astype(np.float32)
    t = np.stack([np.tanh(f[:, 0] + 0.5 * f[:, 1]), 0.3 * f[:, 2] * f[:, 3], np.sin(f[:, 4])], 1).astype(np.float32)
    return f, t


def test_layout_constants_match_the_library(gpu):
    assert gpu.dll.rphys_ext_model_num_params() == ref.N_PARAMS


def test_forward_matches_reference(gpu):
    m = gpu.model(seed=7)
    w = m.weights()
    assert np.all(w[ref.W1:ref.B1].reshape(128, 32)[:, 24:] == 0)
    f, _ = _data(1000, 1)                      # not a multiple of 128: padded rows are ignored
    got = m.predict(f)
    want, _ = ref.forward(w, f)
    err = np.abs(got - want).max() / max(1e-3, np.abs(want).max())
    assert err < 5e-3, err


def test_gradients_match_reference(gpu):
    m = gpu.model(seed=3)
    w = m.weights()
    f, t = _data(512, 2)
    g, loss = m.gradients(f, t)
    g_ref, loss_ref = ref.gradients(w, f, t)
    assert abs(loss - loss_ref) <= 1e-3 * max(1.0, loss_ref)
    for name, a, b in [("W1", ref.W1, ref.B1), ("b1", ref.B1, ref.W2), ("W2", ref.W2, ref.B2), ("W3", ref.W3, ref.B3),
                       ("W4", ref.W4, ref.B4), ("b4", ref.B4, ref.N_PARAMS)]:
        x, y = g[a:b], g_ref[a:b]
        rel = np.linalg.norm(x - y) / max(1e-12, np.linalg.norm(y))
        assert rel < 2e-2, (name, rel)


def test_training_lowers_the_loss(gpu):
    m = gpu.model(seed=5)
    f, t = _data(16384, 4)
    _, l0 = m.gradients(f[:2048], t[:2048])
    m.train(f, t, epochs=4, batch=1024, lr=2e-3)
    _, l1 = m.gradients(f[:2048], t[:2048])
    assert l1 < 0.5 * l0, (l0, l1)
    # determinism: the same seed and data give the same weights
    m2 = gpu.model(seed=5)
    m2.train(f, t, epochs=4, batch=1024, lr=2e-3)
    assert np.array_equal(m.weights(), m2.weights())
