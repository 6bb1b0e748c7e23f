"""Command-line interface: ``python -m quicktex_b200 encode|decode ...``.

The commands, options and defaults are the reference's
(quicktex/cli/__init__.py, encode.py, decode.py); the work runs batched on the
GPU: ``encode`` builds the mip chains of all input images on the device and
encodes every level of every file in one persistent launch; ``decode`` decodes
all files in one launch and flips them on the device."""

import click

from .decode import decode
from .encode import encode


@click.group()
@click.version_option(package_name="quicktex_b200", version="0.1.0")
def main():
    """Encode and Decode various image formats"""


main.add_command(encode)
main.add_command(decode)
