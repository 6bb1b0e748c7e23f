"""CPU: the resize arithmetic of the GPU kernels, restated here in numpy, is
byte-identical to Pillow's BILINEAR resize (resize_no_premultiply); and
mip_sizes matches the reference's chain rules.

The restatement mirrors csrc/qt_resize.cu step for step (taps in double, 22-bit
fixed-point weights, horizontal then vertical 8-bit passes), so this pins the
algorithm that the GPU tests then check on the device against Pillow itself."""

import math

import numpy as np
import pytest

from quicktex_b200.image_utils import mip_sizes, resize_no_premultiply

PB = 22


def taps(n_in, n_out):
    scale = float(np.float32(n_in) - np.float32(0.0)) / n_out
    fs = max(scale, 1.0)
    support = fs
    ksize = int(math.ceil(support)) * 2 + 1
    out = []
    for xx in range(n_out):
        center = 0.0 + (xx + 0.5) * scale
        ss = 1.0 / fs
        xmin = max(int(center - support + 0.5), 0)
        xmax = min(int(center + support + 0.5), n_in) - xmin
        k, ww = [], 0.0
        for x in range(xmax):
            d = (x + xmin - center + 0.5) * ss
            d = -d if d < 0 else d
            w = 1.0 - d if d < 1.0 else 0.0
            k.append(w)
            ww += w
        if ww != 0.0:
            k = [v / ww for v in k]
        kk = [int(-0.5 + v * (1 << PB)) if v < 0 else int(0.5 + v * (1 << PB)) for v in k]
        out.append((xmin, kk))
    return out, ksize


def apply(rows, taps_):
    """rows: (n_in, m, 4) uint8 -> (n_out, m, 4) along axis 0."""
    res = np.empty((len(taps_),) + rows.shape[1:], np.uint8)
    src = rows.astype(np.int64)
    for o, (xmin, kk) in enumerate(taps_):
        s = np.full(rows.shape[1:], 1 << (PB - 1), np.int64)
        for t, c in enumerate(kk):
            s += src[xmin + t] * c
        res[o] = np.clip(s >> PB, 0, 255)
    return res


def resize_restated(rgba, dw, dh):
    h, w = rgba.shape[:2]
    if (dw, dh) == (w, h):
        return rgba.copy()
    th, _ = taps(w, dw)
    tv, _ = taps(h, dh)
    img = rgba
    if dw != w:
        y0 = tv[0][0]
        y1 = tv[-1][0] + len(tv[-1][1])
        img = apply(img[y0:y1].transpose(1, 0, 2), th).transpose(1, 0, 2)
        tv = [(xmin - y0, kk) for xmin, kk in tv]
    if dh != h:
        img = apply(img, tv)
    return img


@pytest.mark.parametrize("w,h,dw,dh", [(37, 21, 18, 10), (37, 21, 1, 1), (64, 64, 32, 32), (64, 64, 2, 2),
                                        (5, 130, 2, 65), (130, 1, 65, 1), (1, 9, 1, 4), (63, 63, 31, 31),
                                        (17, 33, 33, 17), (100, 7, 3, 3)])
def test_restated_resize_matches_pillow(w, h, dw, dh):
    from PIL import Image

    rng = np.random.default_rng(w * 1000 + h)
    rgba = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
    ref = np.asarray(resize_no_premultiply(Image.fromarray(rgba, "RGBA"), (dw, dh)))
    assert np.array_equal(resize_restated(rgba, dw, dh), ref)


def test_mip_sizes():
    assert mip_sizes((37, 21)) == [(37, 21), (18, 10), (9, 5), (4, 2), (2, 1), (1, 1)]
    assert mip_sizes((64, 64), 3) == [(64, 64), (32, 32), (16, 16)]
    assert mip_sizes((1, 1)) == [(1, 1)]
    assert mip_sizes((8, 1), 10) == [(8, 1), (4, 1), (2, 1), (1, 1)]
    with pytest.raises(AssertionError):
        mip_sizes((0, 4))
