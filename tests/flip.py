"""LDR-FLIP image difference, restated in numpy from its publication.

Andersson, Nilsson, Akenine-Möller, Oskarsson, Åström, Fairchild:
"FLIP: A Difference Evaluator for Alternating Images", Proc. ACM Comput.
Graph. Interact. Tech. 3(2), 2020.  Per pixel, a colour error (the images
filtered by contrast sensitivity functions of an opponent colour space, then
the HyAB distance of Hunt-adjusted CIELAB colours, compressed and remapped)
raised to one minus a feature error (differences of edge and point
detector responses on the achromatic channel).  0 means identical; the mean
over pixels is the reported figure.  Inputs are sRGB-encoded in [0, 1].
This module is test infrastructure: it grades rendered frames.
"""
from __future__ import annotations

import numpy as np

PPD = 67.0  # pixels per degree: 0.7 m from a 0.7 m wide 3840-pixel display
QC, PC, PT, QF = 0.7, 0.4, 0.95, 0.5
EDGE_W = 0.082  # degrees
# contrast sensitivity as sums of Gaussians per opponent channel: (a1, b1, a2, b2)
CSF = {"A": (1.0, 0.0047, 0.0, 1e-5), "RG": (1.0, 0.0053, 0.0, 1e-5), "BY": (34.1, 0.04, 13.5, 0.025)}
RGB2XYZ = np.array([[0.4124564, 0.3575761, 0.1804375],
                    [0.2126729, 0.7151522, 0.0721750],
                    [0.0193339, 0.1191920, 0.9503041]])
XYZ2RGB = np.linalg.inv(RGB2XYZ)
WHITE = RGB2XYZ @ np.ones(3)  # D65 white of linear sRGB


def srgb_to_linear(c):
    c = np.asarray(c, np.float64)
    return np.where(c <= 0.04045, c / 12.92, ((c + 0.055) / 1.055) ** 2.4)


def _xyz(rgb):
    return rgb @ RGB2XYZ.T


def _ycxcz(xyz):
    x, y, z = (xyz[..., k] / WHITE[k] for k in range(3))
    return np.stack([116.0 * y - 16.0, 500.0 * (x - y), 200.0 * (y - z)], axis=-1)


def _ycxcz_to_xyz(v):
    y = (v[..., 0] + 16.0) / 116.0
    x = v[..., 1] / 500.0 + y
    z = y - v[..., 2] / 200.0
    return np.stack([x * WHITE[0], y * WHITE[1], z * WHITE[2]], axis=-1)


def _lab(xyz):
    def f(t):
        d = 6.0 / 29.0
        return np.where(t > d ** 3, np.cbrt(t), t / (3 * d * d) + 4.0 / 29.0)
    fx, fy, fz = (f(xyz[..., k] / WHITE[k]) for k in range(3))
    return np.stack([116.0 * fy - 16.0, 500.0 * (fx - fy), 200.0 * (fy - fz)], axis=-1)


def _hunt(lab):
    return np.stack([lab[..., 0], 0.01 * lab[..., 0] * lab[..., 1], 0.01 * lab[..., 0] * lab[..., 2]], axis=-1)


def _hyab(a, b):
    d = a - b
    return np.abs(d[..., 0]) + np.sqrt(d[..., 1] ** 2 + d[..., 2] ** 2)


def _convolve(img, k):
    """Separable-free 2D correlation with edge replication."""
    r = k.shape[0] // 2
    p = np.pad(img, ((r, r), (r, r)), mode="edge")
    out = np.zeros_like(img)
    for i in range(k.shape[0]):
        for j in range(k.shape[1]):
            out += k[i, j] * p[i:i + img.shape[0], j:j + img.shape[1]]
    return out


def _csf_kernel(a1, b1, a2, b2):
    sd = np.sqrt(max(b1, b2) / (2.0 * np.pi ** 2))
    r = int(np.ceil(3.0 * sd * PPD))
    x = np.arange(-r, r + 1) / PPD
    d2 = x[:, None] ** 2 + x[None, :] ** 2
    g = a1 * np.sqrt(np.pi / b1) * np.exp(-np.pi ** 2 * d2 / b1)
    if a2 > 0:
        g = g + a2 * np.sqrt(np.pi / b2) * np.exp(-np.pi ** 2 * d2 / b2)
    return g / g.sum()


def _feature_kernels():
    sd = 0.5 * EDGE_W * PPD
    r = int(np.ceil(3.0 * sd))
    x = np.arange(-r, r + 1, dtype=np.float64)
    X, Y = np.meshgrid(x, x)  # X varies along columns
    g = np.exp(-(X ** 2 + Y ** 2) / (2 * sd * sd))
    edge = -X * g
    point = (X ** 2 / (sd * sd) - 1.0) * g

    def normalise(k):  # positive and negative lobes each of weight one
        pos, neg = k.clip(min=0), k.clip(max=0)
        return pos / pos.sum() + neg / -neg.sum()
    return normalise(edge), normalise(point)


def _features(y):
    ke, kp = _feature_kernels()
    ex, ey = _convolve(y, ke), _convolve(y, ke.T)
    px, py = _convolve(y, kp), _convolve(y, kp.T)
    return np.sqrt(ex * ex + ey * ey), np.sqrt(px * px + py * py)


def flip_map(reference, test):
    """Per-pixel LDR-FLIP of two (H, W, 3) sRGB images in [0, 1]."""
    ref = np.clip(np.asarray(reference, np.float64), 0.0, 1.0)
    tst = np.clip(np.asarray(test, np.float64), 0.0, 1.0)
    # colour pipeline
    filt = []
    for img in (ref, tst):
        v = _ycxcz(_xyz(srgb_to_linear(img)))
        f = np.stack([_convolve(v[..., c], _csf_kernel(*CSF[k])) for c, k in enumerate(("A", "RG", "BY"))], axis=-1)
        lin = np.clip(_ycxcz_to_xyz(f) @ XYZ2RGB.T, 0.0, 1.0)
        filt.append(_hunt(_lab(_xyz(lin))))
    green = _hunt(_lab(_xyz(np.array([0.0, 1.0, 0.0]))))
    blue = _hunt(_lab(_xyz(np.array([0.0, 0.0, 1.0]))))
    cmax = _hyab(green, blue) ** QC
    dc = _hyab(filt[0], filt[1]) ** QC
    knee = PC * cmax
    dc = np.where(dc < knee, PT / knee * dc, PT + (dc - knee) / (cmax - knee) * (1.0 - PT))
    # feature pipeline on the achromatic channel, normalised to [0, 1]
    fr = _features((_ycxcz(_xyz(srgb_to_linear(ref)))[..., 0] + 16.0) / 116.0)
    ft = _features((_ycxcz(_xyz(srgb_to_linear(tst)))[..., 0] + 16.0) / 116.0)
    df = (np.maximum(np.abs(fr[0] - ft[0]), np.abs(fr[1] - ft[1])) / np.sqrt(2.0)) ** QF
    return dc ** (1.0 - df)


def mean_flip(reference, test) -> float:
    return float(flip_map(reference, test).mean())
