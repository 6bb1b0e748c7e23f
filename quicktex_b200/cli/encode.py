"""``encode``: images to DDS files (quicktex/cli/encode.py), all files batched."""

import os

import click

from . import common


def _run(requests_for, flip, remove, suffix, output, filenames):
    """Open every input, build its request, encode them all (one launch per batch), write the files."""
    from PIL import Image

    from .. import dds

    filenames = [f for f in filenames if not f.endswith(".dds")]
    pairs = common.path_pairs(filenames, output, suffix, ".dds")
    reqs = [requests_for(Image.open(p), flip) for p, _ in pairs]
    files = dds.encode_many(reqs)
    with click.progressbar(list(zip(pairs, files)), show_eta=False, show_pos=True,
                           item_show_func=lambda x: str(x[0][0]) if x else "") as bar:
        for (inpath, outpath), f in bar:
            f.save(outpath)
            if remove:
                os.remove(inpath)


def _common_options(f):
    f = click.argument("filenames", nargs=-1, type=click.Path(exists=True, readable=True, dir_okay=False))(f)
    f = click.option("-o", "--output", type=click.Path(writable=True), default=None,
                     help="Output file or directory. If outputting to a file, input filenames must be only a single "
                          "item. By default, files are decoded in place.")(f)
    f = click.option("-s", "--suffix", type=str, default="",
                     help="Suffix to append to output file(s). Ignored if output is a single file.")(f)
    f = click.option("-r", "--remove", is_flag=True, help="Remove input images after converting.")(f)
    f = click.option("-f/-F", "--flip/--no-flip", default=True, show_default=True,
                     help="Vertically flip image before converting.")(f)
    return f


def _level(f):
    return click.option("-l", "--level", type=click.IntRange(0, 18), default=18,
                        help="Quality level to use. Higher values = higher quality, but slower.")(f)


def _bc1_modes(f, prefix=""):
    f = click.option("-3/-4", "--3color/--4color", "threecolor", default=True,
                     help=prefix + "Enable 3-color mode for non-black pixels. Higher quality, but slightly slower.")(f)
    f = click.option("-b/-B", "--black/--no-black",
                     help=prefix + "Enable 3-color mode for blocks containing black or very dark pixels. --3color must "
                          "also be enabled for this to work. (Important: engine/shader MUST ignore decoded texture "
                          "alpha if this flag is enabled!)")(f)
    return f


def _bc1_encoder(level, black, threecolor):
    from ..s3tc.bc1 import BC1Encoder

    cm = BC1Encoder.ColorMode
    mode = cm.FourColor if not threecolor else (cm.ThreeColor if not black else cm.ThreeColorBlack)
    return BC1Encoder(level, mode)


@click.group()
def encode():
    """Encode images to DDS files of the given format."""


@encode.command("bc1")
@_level
@_bc1_modes
@_common_options
def encode_bc1(level, black, threecolor, flip, remove, suffix, output, filenames):
    """Encode images to BC1 (RGB, no alpha)."""
    from ..dds import EncodeRequest

    enc = _bc1_encoder(level, black, threecolor)
    _run(lambda img, fl: EncodeRequest(img, enc, "DXT1", flip=fl), flip, remove, suffix, output, filenames)


@encode.command("bc3")
@_level
@click.option("-n/-N", "--normal/--no-normal", type=bool, default=False,
              help="Perform a BC3nm swizzle, copying the red channel into the alpha [default: no-normal]")
@_common_options
def encode_bc3(level, normal, flip, remove, suffix, output, filenames):
    """Encode images to BC4 (RGBA, 8-bit interpolated alpha)."""
    from ..dds import EncodeRequest
    from ..s3tc.bc3 import BC3Encoder

    enc = BC3Encoder(level)
    _run(lambda img, fl: EncodeRequest(img, enc, "DXT5", flip=fl, swizzle=normal), flip, remove, suffix, output, filenames)


@encode.command("bc4")
@_common_options
def encode_bc4(flip, remove, suffix, output, filenames):
    """Encode images to BC4 (Single channel, 8-bit interpolated red channel)."""
    from ..dds import EncodeRequest
    from ..s3tc.bc4 import BC4Encoder

    enc = BC4Encoder()
    _run(lambda img, fl: EncodeRequest(img, enc, "ATI1", flip=fl), flip, remove, suffix, output, filenames)


@encode.command("bc5")
@_common_options
def encode_bc5(flip, remove, suffix, output, filenames):
    """Encode images to BC5 (2-channel, 8-bit interpolated red and green channels)."""
    from ..dds import EncodeRequest
    from ..s3tc.bc5 import BC5Encoder

    enc = BC5Encoder()
    _run(lambda img, fl: EncodeRequest(img, enc, "ATI2", flip=fl), flip, remove, suffix, output, filenames)


@encode.command("auto")
@_level
@click.option("-b/-B", "--black/--no-black",
              help="[BC1 only] Enable 3-color mode for blocks containing black or very dark pixels. --3color must also "
                   "be enabled for this to work. (Important: engine/shader MUST ignore decoded texture alpha if this "
                   "flag is enabled!)")
@click.option("-3/-4", "--3color/--4color", "threecolor", default=True,
              help="[BC1 only] Enable 3-color mode for non-black pixels. Higher quality, but slightly slower.")
@_common_options
def encode_auto(level, black, threecolor, flip, remove, suffix, output, filenames):
    """Encode images to BC1 or BC3, with the format chosen based on each image's alpha channel."""
    from ..dds import EncodeRequest
    from ..s3tc.bc3 import BC3Encoder

    bc1_enc, bc3_enc = _bc1_encoder(level, black, threecolor), BC3Encoder(level)
    assert len([f for f in filenames if not f.endswith(".dds")]) > 0

    def request(img, fl):
        has_alpha = "A" in img.mode and any(a > 0 for a in img.getchannel("A").histogram()[:-1])
        return EncodeRequest(img, bc3_enc, "DXT5", flip=fl) if has_alpha else EncodeRequest(img, bc1_enc, "DXT1", flip=fl)

    _run(request, flip, remove, suffix, output, filenames)
