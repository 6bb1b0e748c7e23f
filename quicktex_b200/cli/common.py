"""Shared helpers of the command-line tools (quicktex/cli/common.py)."""

from __future__ import annotations

import pathlib
from typing import List

import click


def decoded_extensions(feature: str = "open") -> List[str]:
    """File extensions of the Pillow formats that support ``feature`` ('open' or 'save')."""
    from PIL import Image

    exts = Image.registered_extensions()  # also loads the format plugins
    formats = getattr(Image, feature.upper()).keys()
    return [e for e, f in exts.items() if f in formats]


def validate_decoded_extension(ctx, param, value) -> str:
    """click callback: a leading dot, and an extension Pillow can open."""
    if value[0] != ".":
        value = "." + value
    valid = decoded_extensions()
    if value not in valid:
        raise click.BadParameter(f"Invalid extension for decoded file. Valid extensions are:\n{valid}")
    return value


def path_pairs(inputs, output, suffix: str, extension: str):
    """(input path, output path) pairs: beside each input (no ``output``), into the
    ``output`` file (one input only), or into the ``output`` directory."""
    if len(inputs) < 1:
        raise click.BadArgumentUsage("No valid input files were provided.")
    ins = [pathlib.Path(i) for i in inputs]
    if not output:
        return [(p, p.with_name(p.stem + suffix + extension)) for p in ins]
    out = pathlib.Path(output)
    if out.is_file():
        if len(inputs) > 1:
            raise click.BadOptionUsage("output", "Output is a single file, but multiple input files were provided.")
        return [(p, out) for p in ins]
    return [(p, out / (p.stem + suffix + extension)) for p in ins]
