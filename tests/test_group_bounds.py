"""The group walk's classification rule (slsimlib_b200/csrc/walk_group.cuh),
restated in numpy: a cell accepted for a whole box of rays is accepted by
every ray in the box, and a cell opened for the box is opened by every ray,
under the per-ray FP64 opening test of the reference (open when
dx^2 + dy^2 < open2, quadTree.h:1090).  Seeded boxes and cells, including
cells on and near the box edges and at distances within the 1e-12 margin of
the threshold."""
import numpy as np


def classify(cx, cy, o2, box):
    xmin, xmax, ymin, ymax = box
    nx = np.where(cx < xmin, xmin - cx, np.where(cx > xmax, cx - xmax, 0.0))
    ny = np.where(cy < ymin, ymin - cy, np.where(cy > ymax, cy - ymax, 0.0))
    fx = np.maximum(np.abs(cx - xmin), np.abs(cx - xmax))
    fy = np.maximum(np.abs(cy - ymin), np.abs(cy - ymax))
    dmin2, dmax2 = nx * nx + ny * ny, fx * fx + fy * fy
    accept = dmin2 >= o2 * (1.0 + 1e-12)
    opened = ~accept & (dmax2 < o2 * (1.0 - 1e-12))
    return accept, opened


def test_box_classification_agrees_with_every_ray():
    rng = np.random.default_rng(123)
    for trial in range(200):
        c = rng.uniform(-1, 1, 2) * 10 ** rng.uniform(-3, 2)
        w = 10 ** rng.uniform(-6, -1, 2)
        box = (c[0], c[0] + w[0], c[1], c[1] + w[1])
        rays = np.stack([rng.uniform(box[0], box[1], 128), rng.uniform(box[2], box[3], 128)], axis=1)
        rays[:4] = [[box[0], box[2]], [box[1], box[3]], [box[0], box[3]], [box[1], box[2]]]  # the corners
        rx, ry = rays[:, 0].copy(), rays[:, 1].copy()
        bx = (rx.min(), rx.max(), ry.min(), ry.max())
        n = 512
        cx = c[0] + rng.normal(0, 1, n) * w.max() * 10 ** rng.uniform(-1, 2)
        cy = c[1] + rng.normal(0, 1, n) * w.max() * 10 ** rng.uniform(-1, 2)
        d2 = (cx[:, None] - rx[None, :]) ** 2 + (cy[:, None] - ry[None, :]) ** 2
        # thresholds placed at, just inside and just outside the rays' extreme distances
        lo, hi = d2.min(axis=1), d2.max(axis=1)
        pick = rng.integers(0, 6, n)
        o2 = np.choose(pick, [lo, hi, lo * (1 + 1e-13), hi * (1 - 1e-13), 0.5 * (lo + hi), hi * 1.5])
        accept, opened = classify(cx, cy, o2, bx)
        ray_open = d2 < o2[:, None]
        assert not np.any(ray_open[accept]), trial       # accepted for the box: no ray opens it
        assert np.all(ray_open[opened]), trial            # opened for the box: every ray opens it
