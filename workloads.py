"""Seeded synthetic RGBA8 textures for the encode/decode workloads.

No public corpus exists for this path, so every workload is generated from
numpy's PCG64 with a fixed seed (``0xB2000000 + workload id``), in the shapes,
sizes and value distributions of the reference benchmark plan:

* ``gradient_noise``   smooth per-channel 2-D gradients + uniform noise in
                       [-8, 8], with 10% of the 4x4 blocks overwritten by one
                       solid colour (512x512 BC1 encode+decode workload).
* ``block_mix``        per-block classes: 40% gradient (random endpoints and
                       direction, +-8 noise), 30% uniform random RGB, 20%
                       two-colour edge (random line), 10% solid (4096x4096 BC1
                       workload; also the colour part of the BC3 workload).
* ``alpha_mix``        per-block alpha classes in equal thirds: binary 0/255
                       half-plane cutout, linear ramp, uniform noise.
* ``normal_map``       tangent-space normals of a sum of 8 Gaussian bumps,
                       x/y mapped to [0, 255], packed (x, y, 0, 255).
* ``mixed_batch``      many textures with log-uniform sizes in [4, 2048],
                       25% forced to a non-multiple of 4, formats
                       BC1:BC3:BC4:BC5 = 4:3:2:1, levels uniform in {0,5,10,18}.
* ``hazard_mix``       adversarial blocks aimed at the encoder's rarely taken
                       branches (greyscale, all-black solid, near-black texels,
                       three-colour+black, RGB-uniform blocks with varying alpha,
                       extreme two-colour and solid blocks); ``hazard_counts``
                       counts the blocks that reach each branch.

All arrays are ``uint8`` of shape ``(h, w, 4)``, row-major RGBA.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

SEED_BASE = 0xB2000000

_YY, _XX = np.mgrid[0:4, 0:4]
_XS = (_XX.reshape(16) - 1.5).astype(np.float32)
_YS = (_YY.reshape(16) - 1.5).astype(np.float32)


def rng_for(workload: int, stream: int = 0) -> np.random.Generator:
    # identical to SeedSequence(SEED_BASE + workload).spawn(stream + 1)[stream], without building the siblings
    ss = np.random.SeedSequence(SEED_BASE + workload, spawn_key=(stream,))
    return np.random.Generator(np.random.PCG64(ss))


def _blocks_to_image(blocks: np.ndarray, bw: int, bh: int, w: int, h: int) -> np.ndarray:
    img = blocks.reshape(bh, bw, 4, 4, 4).transpose(0, 2, 1, 3, 4).reshape(bh * 4, bw * 4, 4)
    return np.ascontiguousarray(img[:h, :w])


def _mix_blocks(rng: np.random.Generator, n: int) -> np.ndarray:
    """(n, 16, 3) uint8 colour blocks drawn from the 40/30/20/10 class mix."""
    cls = rng.choice(4, size=n, p=[0.4, 0.3, 0.2, 0.1])
    c0 = rng.integers(0, 256, size=(n, 3)).astype(np.float32)
    c1 = rng.integers(0, 256, size=(n, 3)).astype(np.float32)
    theta = rng.uniform(0, 2 * np.pi, size=n).astype(np.float32)
    offs = rng.uniform(-1.5, 1.5, size=n).astype(np.float32)
    noise = rng.integers(-8, 9, size=(n, 16, 3)).astype(np.float32)
    rand = rng.integers(0, 256, size=(n, 16, 3)).astype(np.float32)

    proj = np.cos(theta)[:, None] * _XS[None] + np.sin(theta)[:, None] * _YS[None]  # (n,16) in ~[-2.1, 2.1]
    t = np.clip(proj / 4.24 + 0.5, 0.0, 1.0)
    grad = c0[:, None, :] + (c1 - c0)[:, None, :] * t[:, :, None] + noise
    edge = np.where((proj > offs[:, None])[:, :, None], c1[:, None, :], c0[:, None, :])
    solid = np.broadcast_to(c0[:, None, :], (n, 16, 3))

    out = np.empty((n, 16, 3), np.float32)
    for k, src in enumerate((grad, rand, edge, solid)):
        m = cls == k
        out[m] = src[m]
    return np.clip(np.rint(out), 0, 255).astype(np.uint8)


def _alpha_blocks(rng: np.random.Generator, n: int) -> np.ndarray:
    """(n, 16) uint8 alpha blocks: cutout / ramp / noise in equal thirds."""
    cls = rng.integers(0, 3, size=n)
    theta = rng.uniform(0, 2 * np.pi, size=n).astype(np.float32)
    offs = rng.uniform(-1.5, 1.5, size=n).astype(np.float32)
    a0 = rng.integers(0, 256, size=n).astype(np.float32)
    a1 = rng.integers(0, 256, size=n).astype(np.float32)
    noise = rng.integers(0, 256, size=(n, 16)).astype(np.float32)
    proj = np.cos(theta)[:, None] * _XS[None] + np.sin(theta)[:, None] * _YS[None]
    cut = np.where(proj > offs[:, None], 255.0, 0.0)
    t = np.clip(proj / 4.24 + 0.5, 0.0, 1.0)
    ramp = a0[:, None] + (a1 - a0)[:, None] * t
    out = np.where((cls == 0)[:, None], cut, np.where((cls == 1)[:, None], ramp, noise))
    return np.clip(np.rint(out), 0, 255).astype(np.uint8)


def block_mix(w: int, h: int, workload: int = 2, stream: int = 0, with_alpha: bool = False) -> np.ndarray:
    rng = rng_for(workload, stream)
    bw, bh = (w + 3) // 4, (h + 3) // 4
    n = bw * bh
    blocks = np.empty((n, 16, 4), np.uint8)
    step = 1 << 18
    for s in range(0, n, step):
        e = min(n, s + step)
        blocks[s:e, :, :3] = _mix_blocks(rng, e - s)
        blocks[s:e, :, 3] = _alpha_blocks(rng, e - s) if with_alpha else 255
    return _blocks_to_image(blocks, bw, bh, w, h)


def alpha_mix(w: int, h: int, workload: int = 3, stream: int = 0) -> np.ndarray:
    return block_mix(w, h, workload, stream, with_alpha=True)


def gradient_noise(w: int = 512, h: int = 512, workload: int = 1, stream: int = 0) -> np.ndarray:
    rng = rng_for(workload, stream)
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    base = np.stack([255 * x / max(w - 1, 1), 255 * y / max(h - 1, 1), 255 * (x + y) / max(w + h - 2, 1)], -1)
    noise = rng.integers(-8, 9, size=(h, w, 3)).astype(np.float32)
    img = np.empty((h, w, 4), np.uint8)
    img[..., :3] = np.clip(np.rint(base + noise), 0, 255).astype(np.uint8)
    img[..., 3] = 255
    bw, bh = (w + 3) // 4, (h + 3) // 4
    nsolid = int(round(0.1 * bw * bh))
    pick = rng.choice(bw * bh, size=nsolid, replace=False)
    cols = rng.integers(0, 256, size=(nsolid, 3)).astype(np.uint8)
    for b, c in zip(pick, cols):
        by, bx = divmod(int(b), bw)
        img[by * 4:by * 4 + 4, bx * 4:bx * 4 + 4, :3] = c
    return img


def normal_map(w: int, h: int, workload: int = 3, stream: int = 1) -> np.ndarray:
    rng = rng_for(workload, stream)
    cx = rng.uniform(0, w, 8)
    cy = rng.uniform(0, h, 8)
    sig = rng.uniform(w / 32, w / 4, 8)
    amp = rng.uniform(-1, 1, 8) * sig  # slopes of order one
    ys = np.arange(h, dtype=np.float32)
    xs = np.arange(w, dtype=np.float32)
    img = np.empty((h, w, 4), np.uint8)
    img[..., 2] = 0
    img[..., 3] = 255
    step = max(1, (1 << 24) // max(w, 1))
    for r0 in range(0, h, step):
        # central differences need one extra row above and below
        yy = np.arange(max(r0 - 1, 0), min(r0 + step + 1, h), dtype=np.float32)
        hf = np.zeros((len(yy), w), np.float32)
        for k in range(8):
            gx = np.exp(-((xs - cx[k]) ** 2) / (2 * sig[k] ** 2)).astype(np.float32)
            gy = np.exp(-((yy - cy[k]) ** 2) / (2 * sig[k] ** 2)).astype(np.float32)
            hf += np.float32(amp[k]) * gy[:, None] * gx[None, :]
        dx = np.gradient(hf, axis=1)
        dy = np.gradient(hf, axis=0) if len(yy) > 1 else np.zeros_like(hf)
        nz = np.ones_like(hf)
        norm = np.sqrt(dx * dx + dy * dy + nz)
        nx, ny = -dx / norm, -dy / norm
        lo = r0 - int(yy[0])
        rows = min(step, h - r0)
        img[r0:r0 + rows, :, 0] = np.clip(np.rint((nx[lo:lo + rows] + 1) * 127.5), 0, 255).astype(np.uint8)
        img[r0:r0 + rows, :, 1] = np.clip(np.rint((ny[lo:lo + rows] + 1) * 127.5), 0, 255).astype(np.uint8)
    del ys
    return img


FORMATS = ("bc1", "bc3", "bc4", "bc5")
LEVELS = (0, 5, 10, 18)


@dataclasses.dataclass
class BatchItem:
    fmt: str
    level: int
    width: int
    height: int
    seed_stream: int

    def texture(self) -> np.ndarray:
        if self.fmt == "bc3":
            return alpha_mix(self.width, self.height, workload=4, stream=self.seed_stream)
        return block_mix(self.width, self.height, workload=4, stream=self.seed_stream)


def mixed_batch(count: int = 10000, workload: int = 4, max_side: int = 2048) -> list[BatchItem]:
    """Descriptors of the mixed-size batch; textures are generated lazily per item."""
    rng = rng_for(workload, 10**6)
    lo, hi = math.log(4), math.log(max_side)
    # log-uniform sides snapped to the 4-texel grid; a quarter are then pushed off it
    ws = np.clip(4 * np.rint(np.exp(rng.uniform(lo, hi, count)) / 4), 4, max_side).astype(int)
    hs = np.clip(4 * np.rint(np.exp(rng.uniform(lo, hi, count)) / 4), 4, max_side).astype(int)
    ragged = rng.random(count) < 0.25
    bump = rng.integers(1, 4, count)
    which = rng.integers(0, 2, count)
    fmts = rng.choice(4, size=count, p=[0.4, 0.3, 0.2, 0.1])
    levels = rng.choice(4, size=count)
    items = []
    for i in range(count):
        w, h = int(ws[i]), int(hs[i])
        if ragged[i]:  # force one side off the 4-texel grid
            if which[i] == 0:
                w = (w // 4) * 4 + int(bump[i])
                w = w - 4 if w > max_side else w
            else:
                h = (h // 4) * 4 + int(bump[i])
                h = h - 4 if h > max_side else h
        items.append(BatchItem(FORMATS[int(fmts[i])], LEVELS[int(levels[i])], w, h, i))
    return items


class MixedBatchPools:
    """Texel sources for the mixed batch: every texture is a window, at a seeded
    offset, of one of two pre-generated 4096x4096 pools (block mix; block mix
    with the alpha mix for BC3), so 10,000 textures cost two pool generations."""

    def __init__(self, workload: int = 4, side: int = 4096):
        self.side = side
        self.rgb = block_mix(side, side, workload=workload, stream=1)
        self.rgba = alpha_mix(side, side, workload=workload, stream=2)
        self.rng = rng_for(workload, 3)

    def texture(self, item: BatchItem) -> np.ndarray:
        pool = self.rgba if item.fmt == "bc3" else self.rgb
        y0 = int(self.rng.integers(0, self.side - item.height + 1))
        x0 = int(self.rng.integers(0, self.side - item.width + 1))
        return np.ascontiguousarray(pool[y0:y0 + item.height, x0:x0 + item.width])


# ---------------------------------------------------------------------------
# adversarial blocks for the encoder's rarely taken branches
# ---------------------------------------------------------------------------
HAZARD_CLASSES = ("grey_narrow", "grey_wide", "black_solid", "near_black_mix", "near_black_edge", "grey_plus_black",
                  "rgb_uniform_alpha", "two_colour_extreme", "solid_extreme", "dark_solid")
_EXTREMES = np.array([0, 1, 2, 3, 4, 5, 7, 8, 127, 128, 250, 253, 254, 255])


def _hazard_blocks(rng: np.random.Generator, cls: np.ndarray) -> np.ndarray:
    """(n, 16, 4) uint8 RGBA blocks; block k drawn from HAZARD_CLASSES[cls[k]]."""
    n = len(cls)
    out = np.empty((n, 16, 4), np.uint8)
    out[..., 3] = 255
    for k, name in enumerate(HAZARD_CLASSES):
        idx = np.nonzero(cls == k)[0]
        m = len(idx)
        if m == 0:
            continue
        b = np.empty((m, 16, 4), np.int64)
        b[..., 3] = 255
        if name == "grey_narrow":  # greyscale, two adjacent levels: max.r - min.r == 1 (< 2), never solid
            base = rng.integers(0, 255, m)
            v = base[:, None] + rng.integers(0, 2, (m, 16))
            v[:, 0], v[:, 1] = base, base + 1
            b[..., 0] = b[..., 1] = b[..., 2] = v
        elif name == "grey_wide":  # greyscale spanning >= 2 levels
            lo = rng.integers(0, 250, m)[:, None]
            hi = np.minimum(255, lo + 2 + rng.integers(0, 120, m)[:, None])
            v = lo + np.floor(rng.random((m, 16)) * (hi - lo + 1)).astype(np.int64)
            v[:, 3], v[:, 12] = lo[:, 0], hi[:, 0]
            b[..., 0] = b[..., 1] = b[..., 2] = v
        elif name == "black_solid":  # every texel (0, 0, 0, a)
            b[..., :3] = 0
            b[..., 3] = np.where(rng.random(m) < 0.25, rng.integers(0, 256, m), 255)[:, None]
        elif name == "near_black_mix":  # (r|g|b) < 4 texels among bright ones: the 3-colour+black trial
            dark = rng.integers(0, 4, (m, 16, 3))
            bright = rng.integers(0, 256, (m, 16, 3))
            bright[:, 0] = np.maximum(bright[:, 0], 64)
            is_dark = rng.random((m, 16)) < rng.uniform(0.15, 0.7, m)[:, None]
            is_dark[:, 0], is_dark[:, 1] = True, False
            b[..., :3] = np.where(is_dark[..., None], dark, bright)
        elif name == "near_black_edge":  # channels straddling the (r|g|b) < 4 rule: 0..7
            b[..., :3] = rng.integers(0, 8, (m, 16, 3))
            b[:, 0, :3] = rng.integers(0, 4, (m, 3))
            b[:, 1, :3] = [4, 0, 0]
        elif name == "grey_plus_black":  # greyscale bright texels plus black ones, texel (0,0) black
            lo = rng.integers(4, 200, m)[:, None]
            v = lo + rng.integers(0, rng.integers(1, 56, m)[:, None] + 1, (m, 16))
            v = np.minimum(v, 255)
            b[..., 0] = b[..., 1] = b[..., 2] = v
            is_dark = rng.random((m, 16)) < 0.4
            is_dark[:, 0], is_dark[:, 1] = True, False
            b[..., :3] = np.where(is_dark[..., None], rng.integers(0, 4, (m, 16, 3)), b[..., :3])
        elif name == "rgb_uniform_alpha":  # one RGB colour, alpha varying: not a solid block
            b[..., :3] = rng.integers(0, 256, (m, 1, 3))
            b[..., 3] = rng.integers(0, 256, (m, 16))
            b[:, 0, 3], b[:, 1, 3] = 0, 255
        elif name == "two_colour_extreme":  # two colours from extreme channel values, random partition
            c = _EXTREMES[rng.integers(0, len(_EXTREMES), (m, 2, 3))]
            c[:, 1, 0] = np.where((c[:, 0] == c[:, 1]).all(1), 255 - c[:, 0, 0], c[:, 1, 0])
            sel = rng.random((m, 16)) < rng.uniform(0.1, 0.9, m)[:, None]
            sel[:, 0], sel[:, 1] = False, True
            b[..., :3] = np.where(sel[..., None], c[:, 1][:, None, :], c[:, 0][:, None, :])
        elif name == "solid_extreme":  # solid blocks of extreme channel values
            b[..., :3] = _EXTREMES[rng.integers(0, len(_EXTREMES), (m, 1, 3))]
        elif name == "dark_solid":  # solid, not black, small channels
            c = rng.integers(0, 8, (m, 1, 3))
            c[:, 0, 2] = np.where((c[:, 0] == 0).all(1), 1, c[:, 0, 2])
            b[..., :3] = c
        out[idx] = np.clip(b, 0, 255).astype(np.uint8)
    return out


def hazard_mix(w: int = 512, h: int = 384, workload: int = 11, stream: int = 0) -> np.ndarray:
    """RGBA8 texture of adversarial blocks: classes of HAZARD_CLASSES in equal shares
    (round-robin over a seeded permutation of the block positions)."""
    rng = rng_for(workload, stream)
    bw, bh = (w + 3) // 4, (h + 3) // 4
    n = bw * bh
    cls = (rng.permutation(n) % len(HAZARD_CLASSES)).astype(np.int64)
    return _blocks_to_image(_hazard_blocks(rng, cls), bw, bh, w, h)


def hazard_counts(img: np.ndarray) -> dict:
    """Blocks of a block-aligned RGBA8 texture that reach each rarely taken branch of
    BC1Encoder::EncodeBlock (BC1Encoder.cpp:261-342):

      grey_narrow     greyscale, not solid, max.r - min.r < 2 (FindEndpoints :476-484)
      grey_wide       greyscale, not solid, max.r - min.r >= 2 (:485-493)
      black_solid     solid with r = g = b = 0 (WriteBlockSolid's all-black rule, :349-353)
      tcb_trial       has_black and not max.IsBlack(): the 3-colour+black trial (:327)
      near_black      holds a texel with (r|g|b) in {3, 4}, either side of IsBlack (Color.h:82)
      grey_ignoring_black  greyscale over its non-black texels but with a black one:
                      the greyscale branch inside the 3-colour+black trial
      rgb_uniform_alpha_varies  one RGB colour, not solid (IsSingleColor compares RGBA)
    """
    hh, ww = img.shape[:2]
    bl = img.reshape(hh // 4, 4, ww // 4, 4, 4).transpose(0, 2, 1, 3, 4).reshape(-1, 16, 4).astype(np.int64)
    rgb = bl[..., :3]
    solid = (bl == bl[:, :1]).all((1, 2))
    grey = ((rgb[..., 0] == rgb[..., 1]) & (rgb[..., 0] == rgb[..., 2])).all(1)
    rng_r = rgb[..., 0].max(1) - rgb[..., 0].min(1)
    ored = rgb[..., 0] | rgb[..., 1] | rgb[..., 2]
    is_black = ored < 4
    mx = rgb.max(1)
    max_black = (mx[:, 0] | mx[:, 1] | mx[:, 2]) < 4
    nb_grey = np.where(is_black, True, (rgb[..., 0] == rgb[..., 1]) & (rgb[..., 0] == rgb[..., 2])).all(1)
    rgb_uni = (rgb == rgb[:, :1]).all((1, 2))
    return {
        "grey_narrow": int((grey & ~solid & (rng_r < 2)).sum()),
        "grey_wide": int((grey & ~solid & (rng_r >= 2)).sum()),
        "black_solid": int((solid & (ored[:, 0] == 0)).sum()),
        "tcb_trial": int((~solid & is_black.any(1) & ~max_black).sum()),
        "near_black": int((~solid & ((ored == 3) | (ored == 4)).any(1)).sum()),
        "grey_ignoring_black": int((~solid & ~grey & nb_grey & is_black.any(1) & ~max_black).sum()),
        "rgb_uniform_alpha_varies": int((rgb_uni & ~solid).sum()),
    }
