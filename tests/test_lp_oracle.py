"""The proposal network's CPU oracle checked against itself: its analytic gradients against
central finite differences of its loss in exact float64 arithmetic (no bf16 rounding), and its
bf16 rounding against the definition (nearest even)."""
import numpy as np

from oracle import lp_oracle as lo


def _setup(seed=3, F=2, mbw=3, mbh=2):
    rng = np.random.default_rng(seed)
    p = np.zeros(lo.param_count())
    layers_w = []
    o = 0
    for l in range(lo.LAYERS):
        n = lo.wcount(l)
        p[o:o + n] = rng.normal(0, np.sqrt(2.0 / (9 * lo.cin(l))), n)
        o += n
        p[o:o + lo.C] = rng.normal(0, 0.05, lo.C)
        o += lo.C
    p[o:] = rng.normal(0, 0.2, lo.param_count() - o)
    x0 = rng.normal(0, 0.7, (F, 4 * mbh, 4 * mbw, lo.CIN0))
    hints = [(int(rng.integers(-20, 20)), int(rng.integers(-20, 20))) for _ in range(F)]
    labels = rng.integers(-24, 24, (F, mbw * mbh, 2))
    return p, x0, hints, labels, mbw, mbh


def test_oracle_gradients_match_finite_differences():
    p, x0, hints, labels, mbw, mbh = _setup()
    loss, g = lo.loss_and_grads(p, x0, hints, labels, mbw, mbh, rounding=False)
    rng = np.random.default_rng(7)
    idx = rng.choice(len(p), 60, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = lo.loss_and_grads(q, x0, hints, labels, mbw, mbh, rounding=False)
        q[i] -= 2 * eps
        lm, _ = lo.loss_and_grads(q, x0, hints, labels, mbw, mbh, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), (i, fd, g[i])
    assert np.isfinite(loss)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5, 0.0], np.float32)
    got = lo.bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0            # halfway, rounds to even
    assert got[2] == 1.0 + 2 ** -6  # halfway, rounds to even (up)
    assert got[3] == 1.0
    assert got[4] == -2.5 and got[5] == 0.0


def test_hint_search_finds_a_known_translation():
    rng = np.random.default_rng(1)
    base = rng.integers(0, 256, (96, 160)).astype(np.uint8)
    base = np.kron(base[::4, ::4], np.ones((4, 4), np.uint8))[:96, :160]  # smooth enough to align
    cur = np.roll(base, (5, -12), axis=(0, 1))
    gx, gy = lo.hint_search(cur, base, 32)
    assert (gx, gy) == (12, -5)
