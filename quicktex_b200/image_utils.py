"""Mip-chain helpers: the interface of quicktex's ``image_utils`` module
(quicktex/image_utils.py), plus the same resize on the GPU.

``mip_sizes`` and ``resize_no_premultiply`` behave as the reference's (the
latter is Pillow's BILINEAR resize of the RGB and alpha bands separately, on the
CPU). ``resize_device`` does that resize on device buffers through
``qt_resize_bilinear_device``, byte-identical to Pillow's.
"""

from __future__ import annotations

import ctypes
import math
from typing import List, Optional, Tuple

from . import capi


def mip_sizes(dimensions: Tuple[int, int], mip_count: Optional[int] = None) -> List[Tuple[int, int]]:
    """Sizes of a mip chain starting at ``dimensions``: each level halves both
    sides, rounding down, never below 1 (quicktex/image_utils.py:9-37). Without
    ``mip_count`` the chain runs to 1x1; it also stops early at 1x1."""
    assert all(d > 0 for d in dimensions), "Invalid source dimensions"
    if not mip_count:
        mip_count = math.ceil(math.log2(max(dimensions)) + 1)
    assert mip_count > 0, "mip_count must be greater than 0"
    chain = []
    w, h = dimensions
    for _ in range(mip_count):
        chain.append((w, h))
        if w == 1 and h == 1:
            break
        w, h = max(w // 2, 1), max(h // 2, 1)
    return chain


def resize_no_premultiply(image, size: Tuple[int, int]):
    """Pillow BILINEAR resize without premultiplied alpha (quicktex/image_utils.py:40-52)."""
    from PIL import Image

    if image.mode == "RGBA":
        rgb = image.convert("RGB").resize(size, Image.BILINEAR)
        a = image.getchannel("A").resize(size, Image.BILINEAR)
        rgb.putalpha(a)
        return rgb
    return image.resize(size, Image.BILINEAR)


def resize_device(src: int, width: int, height: int, dst: int, new_width: int, new_height: int, stream: int = 0) -> None:
    """``resize_no_premultiply`` of an RGBA8 texture on the GPU: ``src`` and ``dst``
    are device addresses; enqueued on ``stream``."""
    v = ctypes.c_void_p
    capi.check(capi.lib().qt_resize_bilinear_device(v(src), width, height, v(dst), new_width, new_height, v(stream)))
