"""Seeded source / prediction pictures for the DQUANT search tests, built to reach each of its
branches: flat macroblocks beside detail (the adjacency path), sparse bright detail on dark,
smooth bright content with a small residual (the coarser candidates), saturated blue dark detail
(the perceptual priority's boost, so the base MQUANT differs from PQINDEX) and natural texture."""
import numpy as np
def frames(kind, w, h, seed):
    rng = np.random.default_rng(seed)
    mbw, mbh = (w + 15) // 16, (h + 15) // 16
    yy, xx = np.mgrid[0:h, 0:w]
    if kind == "adjacency":
        flat = ((xx // 16 + yy // 16) % 2 == 0)
        y = np.where(flat, 80, rng.integers(0, 256, (h, w)))
    elif kind == "bright_on_dark":
        y = np.full((h, w), 30) + rng.integers(0, 6, (h, w))
        dots = rng.random((h, w)) < 0.06
        y = np.where(dots, 220, y)
        y[:, w // 2:] = 120 + rng.integers(-30, 30, (h, w - w // 2))
    elif kind == "dark_detail":
        y = 26 + 22 * np.sin(xx / 1.3) * np.cos(yy / 1.7) + rng.normal(0, 3, (h, w))
        y[:, : w // 3] = 150
    elif kind == "coarser":
        y = 200 + 20 * np.sin(xx / 9.0) + 15 * np.cos(yy / 7.0)
    else:
        y = 128 + 60 * np.sin(xx / 5.0) * np.cos(yy / 11.0) + rng.normal(0, 8, (h, w))
    y = np.clip(np.rint(y), 0, 255).astype(np.uint8)
    u = np.full((h // 2, w // 2), 128, np.uint8) + rng.integers(0, 3, (h // 2, w // 2)).astype(np.uint8)
    v = np.full((h // 2, w // 2), 128, np.uint8)
    if kind == "dark_detail":  # saturated blue in the dark part: the perceptual priority's boost
        u[:, w // 6:] = 180
        v[:, w // 6:] = 76
    noise = rng.normal(0, {"bright_on_dark": 12.0, "natural": 12.0, "dark_detail": 6.0}.get(kind, 2.5), (h, w))
    py = np.clip(np.rint(y + noise), 0, 255).astype(np.uint8)
    return (y, u, v), (py, u.copy(), v.copy())
