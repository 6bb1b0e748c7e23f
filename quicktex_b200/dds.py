"""DDS files with mip chains: the interface of quicktex's ``dds`` module
(quicktex/dds.py), with the mip chain built and coded on the GPU.

``encode(image, encoder, four_cc, mip_count)`` uploads the image once, resizes
it to every mip level on the device (``qt_resize_bilinear_device``, byte-identical
to the reference's Pillow resize), and encodes all levels in ONE persistent
batch launch. ``DDSFile.decode_all`` decodes every level in one launch as well.
The file bytes equal the reference's ``dds.encode(...).save(...)`` for the same
image and encoder settings (tests check this against files the reference wrote).

The header layout is the DirectX DDS format (magic, 124-byte header, 32-byte
pixel format), written field for field as quicktex/dds.py:161-193 writes it.
"""

from __future__ import annotations

import enum
import os
import struct
import typing

import numpy as np

from . import capi
from . import image_utils
from .s3tc import bc1, bc3, bc4, bc5


class DDSFormat:
    def __init__(self, name: str, texture, encoder, decoder, four_cc: str = None):
        self.four_cc = four_cc
        self.decoder = decoder
        self.encoder = encoder
        self.texture = texture
        self.name = name


dds_formats = [
    DDSFormat("BC1", bc1.BC1Texture, bc1.BC1Encoder, bc1.BC1Decoder, "DXT1"),
    DDSFormat("BC3", bc3.BC3Texture, bc3.BC3Encoder, bc3.BC3Decoder, "DXT5"),
    DDSFormat("BC4", bc4.BC4Texture, bc4.BC4Encoder, bc4.BC4Decoder, "ATI1"),
    DDSFormat("BC5", bc5.BC5Texture, bc5.BC5Encoder, bc5.BC5Decoder, "ATI2"),
]


class PFFlags(enum.IntFlag):
    """DDS_PIXELFORMAT flags."""

    ALPHAPIXELS = 0x1
    ALPHA = 0x2
    FOURCC = 0x4
    RGB = 0x40
    YUV = 0x200
    LUMINANCE = 0x20000


class DDSFlags(enum.IntFlag):
    """DDS_HEADER flags: which members hold valid data."""

    CAPS = 0x1
    HEIGHT = 0x2
    WIDTH = 0x4
    PITCH = 0x8
    PIXEL_FORMAT = 0x1000
    MIPMAPCOUNT = 0x20000
    LINEAR_SIZE = 0x80000
    DEPTH = 0x800000
    TEXTURE = CAPS | HEIGHT | WIDTH | PIXEL_FORMAT


class Caps0(enum.IntFlag):
    """DDS_HEADER caps: surface complexity."""

    COMPLEX = 0x8
    MIPMAP = 0x400000
    TEXTURE = 0x1000


_BLOCK_BYTES = {"BC1": 8, "BC3": 16, "BC4": 8, "BC5": 16}


@typing.final
class DDSFile:
    """A DDS file: header fields and one block texture per mip level."""

    magic = b"DDS "
    extension = "dds"
    header_bytes = 124

    def __init__(self):
        self.flags: DDSFlags = DDSFlags.TEXTURE
        self.size: typing.Tuple[int, int] = (0, 0)
        self.pitch: int = 0
        self.depth: int = 1
        self.mipmap_count: int = 1
        self.pf_flags: PFFlags = PFFlags.FOURCC
        self.four_cc: str = "NONE"
        self.pixel_size: int = 0
        self.pixel_bitmasks: typing.Tuple[int, int, int, int] = (0, 0, 0, 0)
        self.caps: typing.Tuple[Caps0, int, int, int] = (Caps0.TEXTURE, 0, 0, 0)
        self.textures: typing.List = []
        self.format: DDSFormat = DDSFormat("NONE", None, None, None)

    def tobytes(self) -> bytes:
        """The whole file: magic, header, then every level's blocks."""
        head = struct.pack("<7I44x", DDSFile.header_bytes, int(self.flags), self.size[1], self.size[0], self.pitch,
                           self.depth, self.mipmap_count)
        pf = struct.pack("<2I4s5I", 32, int(self.pf_flags), bytes(self.four_cc, "ascii"), self.pixel_size,
                         *self.pixel_bitmasks)
        caps = struct.pack("<4I4x", *[int(c) for c in self.caps])
        out = DDSFile.magic + head + pf + caps
        assert len(out) == 4 + DDSFile.header_bytes, "error writing file: incorrect header size"
        return out + b"".join(bytes(t) for t in self.textures)

    def save(self, path: os.PathLike) -> None:
        with open(path, "wb") as f:
            f.write(self.tobytes())

    def decode(self, mip: int = 0, *args, **kwargs):
        """One level as a PIL image (decoder built from ``args``/``kwargs`` as the reference does)."""
        return self._decode([mip], self.format.decoder(*args, **kwargs))[0]

    def decode_all(self, *args, **kwargs) -> list:
        """Every level as PIL images, decoded in one batch launch."""
        return self._decode(range(len(self.textures)), self.format.decoder(*args, **kwargs))

    def _decode(self, mips, decoder) -> list:
        from PIL import Image

        texs = [self.textures[m] for m in mips]
        item = _decode_item(self.format.name, decoder)
        if item is None:  # a decoder the batch path does not know: one call per level
            raws = [decoder.decode(t) for t in texs]
            return [Image.frombuffer("RGBA", r.size, r.tobytes(), "raw", "RGBA", 0, 1) for r in raws]
        from .batch import Job, run_jobs

        fmt = self.format.name.lower()
        jobs = [Job.decode(fmt, np.frombuffer(bytes(t), np.uint8), t.width, t.height, **item) for t in texs]
        outs = run_jobs(jobs)  # every level in one launch
        return [Image.frombuffer("RGBA", t.size, o, "raw", "RGBA", 0, 1) for t, o in zip(texs, outs)]


def read(path: os.PathLike) -> DDSFile:
    """Parse a DDS file written with a FourCC of DXT1, DXT5, ATI1 or ATI2 (quicktex/dds.py:218-273)."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == DDSFile.magic, "Incorrect magic bytes in DDS file."
    dds = DDSFile()
    (header_bytes,) = struct.unpack_from("<I", data, 4)
    assert header_bytes == DDSFile.header_bytes, "Incorrect DDS header size."
    flags, height, width, pitch, depth, mips = struct.unpack_from("<6I", data, 8)
    dds.flags = DDSFlags(flags)
    dds.size = (width, height)
    dds.pitch, dds.depth, dds.mipmap_count = pitch, depth, mips
    (pf_size,) = struct.unpack_from("<I", data, 76)
    assert pf_size == 32, "Incorrect pixel format size."
    (pf_flags,) = struct.unpack_from("<I", data, 80)
    dds.pf_flags = PFFlags(pf_flags)
    dds.four_cc = data[84:88].decode()
    dds.pixel_size, *masks = struct.unpack_from("<5I", data, 88)
    dds.pixel_bitmasks = tuple(masks)
    dds.caps = struct.unpack_from("<4I", data, 108)
    offset = 4 + DDSFile.header_bytes
    if DDSFlags.DEPTH not in dds.flags:
        dds.depth = 1
    if DDSFlags.MIPMAPCOUNT not in dds.flags:
        dds.mipmap_count = 1
    if PFFlags.FOURCC not in dds.pf_flags:
        dds.four_cc = "NONE"
    if dds.four_cc == "DX10":
        raise NotImplementedError("DX10 headers are not yet supported")
    dds.format = next(entry for entry in dds_formats if entry.four_cc == dds.four_cc)
    dds.textures = []
    for w, h in image_utils.mip_sizes(dds.size, dds.mipmap_count):
        n = ((w + 3) // 4) * ((h + 3) // 4) * _BLOCK_BYTES[dds.format.name]
        chunk = data[offset: offset + n]
        assert len(chunk) == n, "Unexpected end of file"
        dds.textures.append(dds.format.texture.from_bytes(chunk, w, h))
        offset += n
    return dds


def _interp_id(interp) -> int:
    name = type(interp).__name__
    return {"Interpolator": 0, "InterpolatorRound": 1, "InterpolatorNvidia": 2, "InterpolatorAMD": 3}[name]


def _bc1_params(e) -> capi.BC1Params:
    p = capi.BC1Params()
    p.color_mode = int(e.color_mode)
    p.interpolator = _interp_id(e.interpolator)
    p.error_mode = int(e.error_mode)
    p.endpoint_mode = int(e.endpoint_mode)
    p.two_ls_passes, p.two_ep_passes, p.two_cf_passes = int(e.two_ls_passes), int(e.two_ep_passes), int(e.two_cf_passes)
    p.exhaustive = int(e.exhaustive)
    p.search_rounds = int(e.search_rounds)
    p.orderings4, p.orderings3 = (int(x) for x in e.orderings)
    p.power_iterations = int(e.power_iterations)
    return p


def _encode_item(encoder) -> typing.Optional[dict]:
    """Batch settings of a known encoder (``Job.encode`` keywords), else None."""
    if isinstance(encoder, bc1.BC1Encoder):
        return {"fmt": "bc1", "params": _bc1_params(encoder)}
    if isinstance(encoder, bc3.BC3Encoder):
        return {"fmt": "bc3", "params": _bc1_params(encoder.bc1_encoder)}
    if isinstance(encoder, bc4.BC4Encoder):
        return {"fmt": "bc4", "channel": int(encoder.channel)}
    if isinstance(encoder, bc5.BC5Encoder):
        c0, c1 = encoder.channels
        return {"fmt": "bc5", "chan0": int(c0), "chan1": int(c1)}
    return None


def _decode_item(fmt: str, decoder) -> typing.Optional[dict]:
    if fmt == "BC1" and isinstance(decoder, bc1.BC1Decoder):
        return {"interpolator": _interp_id(decoder.interpolator), "write_alpha": bool(decoder.write_alpha)}
    if fmt == "BC3" and isinstance(decoder, bc3.BC3Decoder):
        return {"interpolator": _interp_id(decoder.bc1_decoder.interpolator)}
    if fmt == "BC4" and isinstance(decoder, bc4.BC4Decoder):
        return {"channel": int(decoder.channel)}
    if fmt == "BC5" and isinstance(decoder, bc5.BC5Decoder):
        c0, c1 = decoder.channels
        return {"chan0": int(c0), "chan1": int(c1)}
    return None


class EncodeRequest:
    """One image to encode into a DDS file, as ``dds.encode`` and the command-line
    encoder take it: ``flip`` turns it upside down first (Image.FLIP_TOP_BOTTOM)
    and ``swizzle`` applies the BC3nm swizzle (RGBA = 1, G, G, R) after that."""

    def __init__(self, image, encoder, four_cc: str, mip_count: typing.Optional[int] = None, flip: bool = False,
                 swizzle: bool = False):
        self.image, self.encoder, self.four_cc, self.mip_count = image, encoder, four_cc, mip_count
        self.flip, self.swizzle = flip, swizzle


def _prepare(r: EncodeRequest):
    """CPU side of one request: the texels as dds.encode converts them, and what is
    left for the device to do (flip, swizzle channels). Conversions act on each
    texel alone, so doing them before the flip gives the same texels."""
    from PIL import Image

    image, flip, swz = r.image, r.flip, None
    if r.swizzle:
        if image.mode in ("RGB", "RGBA", "RGBX", "RGBa"):
            swz, mode = (0, 1), "RGBA"
        elif image.mode in ("LA", "La"):
            swz, mode = (0, 3), "RGBA"  # LA -> RGBA is (L, L, L, A): bands 0 and 1 sit at channels 0 and 3
        else:  # other modes: the reference's own steps on the CPU
            if flip:
                image = image.transpose(Image.FLIP_TOP_BOTTOM)
                flip = False
            bands = image.split()
            one = Image.new("L", image.size, 0xFF)
            image = Image.merge("RGBA", (one, bands[1], bands[1], bands[0]))
            mode = "RGBA"
    else:
        mode = "RGBA" if "A" in image.mode else "RGBX"
    image.apply_transparency()
    if image.mode != mode:  # convert() would return an identical copy
        image = image.convert(mode)
    return image, mode, flip, swz


_staging = None


def _pinned(nbytes: int):
    """A pinned host buffer of at least ``nbytes``, reused across calls (callers finish
    their copies before returning)."""
    import torch

    global _staging
    if _staging is None or _staging.numel() < nbytes:
        _staging = torch.empty(max(nbytes, 1 << 24), dtype=torch.uint8).pin_memory()
    return _staging


def encode_many(requests: typing.Sequence[EncodeRequest], max_batch_bytes: int = 2 << 30) -> typing.List[DDSFile]:
    """Encode many images with their mip chains. On the device: each image is
    uploaded once, flipped / swizzled if asked, resized to every level; then the
    levels of all images (up to ``max_batch_bytes`` of texels at a time) are
    encoded in one persistent batch launch."""
    import torch

    from . import RawTexture
    from .batch import Batch, Job, copy_async

    prepared = [_prepare(r) for r in requests]
    out: typing.List[typing.Optional[DDSFile]] = [None] * len(requests)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    align = lambda n: (n + 255) // 256 * 256  # noqa: E731
    pending = []  # (index, sizes, fmt, item)

    def flush():
        if not pending:
            return
        # device layout: packed uploads, then every level's texels, then every level's blocks
        up_off, lv_off, out_off, nu, nl, no = [], [], [], 0, 0, 0
        for _, sizes, fmt, _item, _img in pending:
            bb = _BLOCK_BYTES[fmt.name]
            w0, h0 = sizes[0]
            up_off.append(nu)
            nu += align(w0 * h0 * 4)
            lv_in, lv_out = [], []
            for w, h in sizes:
                lv_in.append(nl)
                lv_out.append(no)
                nl += align(w * h * 4)
                no += align(((w + 3) // 4) * ((h + 3) // 4) * bb)
            lv_off.append(lv_in)
            out_off.append(lv_out)
        stage = _pinned(nu).numpy()
        for (i, sizes, *_rest), o in zip(pending, up_off):
            img, mode = pending_img[i], prepared[i][1]
            raw = np.frombuffer(img.tobytes("raw", mode), np.uint8)
            stage[o: o + raw.size] = raw
        d_up = torch.empty(nu, dtype=torch.uint8, device=dev)
        d_lv = torch.empty(nl, dtype=torch.uint8, device=dev)
        d_out = torch.empty(max(no, 1), dtype=torch.uint8, device=dev)
        d_up.copy_(_staging[:nu], non_blocking=True)  # one upload for all images
        ub, lb, ob, sp = d_up.data_ptr(), d_lv.data_ptr(), d_out.data_ptr(), stream.cuda_stream
        items = []
        for (i, sizes, fmt, item, _img), uo, lv_in, lv_out in zip(pending, up_off, lv_off, out_off):
            _, _mode, flip, swz = prepared[i]
            w0, h0 = sizes[0]
            c0, c1 = swz if swz else (-1, 0)
            capi.check(capi.lib().qt_flip_swizzle_device(capi._vp(ub + uo), w0, h0, capi._vp(lb + lv_in[0]),
                                                        int(flip), c0, c1, capi._vp(sp)))
            for (w, h), off in zip(sizes[1:], lv_in[1:]):  # every level from the (prepared) original
                image_utils.resize_device(lb + lv_in[0], w0, h0, lb + off, w, h, sp)
            kw = {k: v for k, v in item.items() if k != "fmt"}
            for (w, h), a, b in zip(sizes, lv_in, lv_out):
                items.append(Job.encode(item["fmt"], np.zeros(0, np.uint8), w, h, **kw).item(lb + a, ob + b))
        # the result textures first (their storage is pinned host memory), so every level's
        # blocks are copied from the device straight into its texture
        made, copies = [], []
        for (i, sizes, fmt, _item, _img), lv_out in zip(pending, out_off):
            texs = [fmt.texture._uninitialized(w, h) for w, h in sizes]
            for t, o in zip(texs, lv_out):
                copies.append((np.frombuffer(memoryview(t), np.uint8).ctypes.data, ob + o, t.nbytes))
            made.append((i, texs, fmt))
        batch = Batch(dev.index)
        try:
            batch.run(items, sp)  # every level of every image in one persistent launch
            copy_async(np.array(copies, np.uint64).reshape(-1, 3), sp)
            stream.synchronize()
        finally:
            batch.close()
        for i, texs, fmt in made:
            out[i] = _dds_file(texs, requests[i].four_cc, fmt)
        pending.clear()

    pending_img = {}
    held = 0
    for i, (r, (img, mode, flip, swz)) in enumerate(zip(requests, prepared)):
        sizes = image_utils.mip_sizes(img.size, r.mip_count)
        item = _encode_item(r.encoder)
        fmt = next((f for f in dds_formats if item is not None and f.name == item["fmt"].upper()), None)
        if fmt is None:  # an encoder the batch path does not know: the reference's per-level calls
            from PIL import Image

            if flip:
                img = img.transpose(Image.FLIP_TOP_BOTTOM)
            if swz:
                bands = img.split()
                img = Image.merge("RGBA", (Image.new("L", img.size, 0xFF), bands[swz[1]], bands[swz[1]], bands[swz[0]]))
            levels = [img] + [image_utils.resize_no_premultiply(img, s) for s in sizes[1:]]
            texs = [r.encoder.encode(RawTexture.frombytes(lv.tobytes("raw", mode), *lv.size)) for lv in levels]
            out[i] = _dds_file(texs, r.four_cc, None)
            continue
        need = 2 * sum(w * h * 4 for w, h in sizes)
        if pending and held + need > max_batch_bytes:
            flush()
            held = 0
        pending.append((i, sizes, fmt, item, img))
        pending_img[i] = img
        held += need
    flush()
    return out


def _dds_file(textures, four_cc: str, fmt) -> DDSFile:
    """Header fields as quicktex/dds.py:285-303 sets them."""
    dds = DDSFile()
    dds.textures = textures
    dds.flags = DDSFlags.TEXTURE | DDSFlags.LINEAR_SIZE
    caps0 = Caps0.TEXTURE
    if len(textures) > 1:
        dds.flags |= DDSFlags.MIPMAPCOUNT
        caps0 |= Caps0.MIPMAP | Caps0.COMPLEX
    dds.caps = (caps0, 0, 0, 0)
    dds.mipmap_count = len(textures)
    dds.pitch = textures[0].nbytes
    dds.size = textures[0].size
    dds.pf_flags = PFFlags.FOURCC
    dds.four_cc = four_cc
    if fmt is not None:
        dds.format = fmt
    return dds


def encode(image, encoder, four_cc: str, mip_count: typing.Optional[int] = None) -> DDSFile:
    """Encode a PIL image and its mip chain (quicktex/dds.py:275-303): the chain's
    sizes halve down to 1x1 (or ``mip_count`` levels), every level is the
    original resized with BILINEAR filtering, RGB and alpha separately. The
    whole chain is resized on the device and encoded in one batch launch."""
    return encode_many([EncodeRequest(image, encoder, four_cc, mip_count)])[0]


def decode_many(files: typing.Sequence[DDSFile], mip: int = 0, flip: bool = False) -> list:
    """Level ``mip`` of every file as PIL images, with each format's default
    decoder (as ``DDSFile.decode()``): all files in one batch launch, then, with
    ``flip``, turned upside down on the device (the command-line decoder's
    Image.FLIP_TOP_BOTTOM)."""
    import torch
    from PIL import Image

    from .batch import Batch, Job

    if not files:
        return []
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    align = lambda n: (n + 255) // 256 * 256  # noqa: E731
    texs = [f.textures[mip] for f in files]
    jobs = [Job.decode(f.format.name.lower(), np.frombuffer(bytes(t), np.uint8), t.width, t.height,
                       **_decode_item(f.format.name, f.format.decoder())) for f, t in zip(files, texs)]
    in_off, out_off, ni, no = [], [], 0, 0
    for j in jobs:
        in_off.append(ni)
        out_off.append(no)
        ni += align(j.data.nbytes)
        no += align(j.out_bytes)
    h_in = torch.empty(ni, dtype=torch.uint8).pin_memory()
    hn = h_in.numpy()
    for j, o in zip(jobs, in_off):
        hn[o: o + j.data.nbytes] = j.data
    d_in = h_in.to(dev, non_blocking=True)
    d_out = torch.empty(no, dtype=torch.uint8, device=dev)
    d_flip = torch.empty(no, dtype=torch.uint8, device=dev) if flip else d_out
    ib, ob, fb = d_in.data_ptr(), d_out.data_ptr(), d_flip.data_ptr()
    batch = Batch(dev.index)
    try:
        batch.run([j.item(ib + a, ob + b) for j, a, b in zip(jobs, in_off, out_off)], sp)
        if flip:
            for j, b in zip(jobs, out_off):
                capi.check(capi.lib().qt_flip_swizzle_device(capi._vp(ob + b), j.width, j.height, capi._vp(fb + b),
                                                            1, -1, 0, capi._vp(sp)))
        h_out = torch.empty(no, dtype=torch.uint8).pin_memory()  # a pinned download runs at the link's rate
        h_out.copy_(d_flip, non_blocking=True)
        stream.synchronize()
        host = h_out.numpy()
    finally:
        batch.close()
    return [Image.frombuffer("RGBA", (j.width, j.height), host[b: b + j.out_bytes].tobytes(), "raw", "RGBA", 0, 1)
            for j, b in zip(jobs, out_off)]
