"""CPU checks of the learned Newton start's reference net (oracle/guess_ref.py): its
analytic gradient against finite differences, and the BF16 rounding it emulates."""
import numpy as np

import guess_ref as G


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -7, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 0.0],
                 dtype=np.float32)
    r = G.bf16(x)
    # 7 fraction bits: 1 + 2^-7 is representable; 1 + 2^-8 is a tie -> even (1.0);
    # 1 + 3 * 2^-8 is a tie between 1 + 2^-7 and 1 + 2^-6 -> even (1 + 2^-6)
    assert r.tolist() == [1.0, 1.0 + 2.0 ** -7, 1.0, 1.0 + 2.0 ** -6, -2.5, 0.0]


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    w = G.init_weights(5).astype(np.float64)
    s = np.zeros((40, 8))
    s[:, :6] = 0.7 * rng.standard_normal((40, 6))
    s[:, 6] = rng.standard_normal(40)
    s[:, 7] = 1.0
    s[5, 7] = 0.0  # an unusable sample carries no weight

    def loss(wv):
        l, _ = G.loss_and_grad(wv, s, rounding=False)
        return l / s.shape[0]

    _, g = G.loss_and_grad(w, s, rounding=False)
    idx = np.concatenate([rng.choice(np.arange(G.OFF_B1), 12, replace=False),
                          G.OFF_B1 + rng.choice(64, 4, replace=False),
                          G.OFF_W2 + rng.choice(4096, 16, replace=False),
                          G.OFF_B2 + rng.choice(64, 4, replace=False),
                          G.OFF_W3 + rng.choice(64, 6, replace=False), [G.OFF_B3]])
    for i in idx:
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        fd = (loss(wp) - loss(wm)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_samples_from_records_target_definition():
    # equal states: acoustic start exact, no usable target; a shock: target r defined
    rec = np.array([[1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 1.0, 1.0],
                    [1.0, 0.125, 1.0, 0.1, 0.0, 0.0, 0.30313, 4.0]])
    s = G.samples_from_records(rec, 1.4, 1e-20)
    assert s[0, 7] == 0.0
    assert s[1, 7] == 1.0
    f, d2 = G.features(1.0, 0.125, 1.0, 0.1, 0.0, 0.0, 1.4)
    ps = G.acoustic_start(1.0, 0.125, 1.0, 0.1, 0.0, 0.0, 1.4, 1e-20)
    assert np.isclose(s[1, 6], np.log(0.30313 / ps) / d2, rtol=1e-6)
