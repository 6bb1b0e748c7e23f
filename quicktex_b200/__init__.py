"""quicktex_b200 — the S3TC (BC1/BC3/BC4/BC5) encode/decode path of quicktex on
NVIDIA B200 (sm_100a).

The package mirrors the reference's Python interface: ``quicktex_b200.RawTexture``
and ``quicktex_b200.s3tc.{bc1,bc3,bc4,bc5,interpolator}`` hold the classes the
reference exposes under ``quicktex`` and ``quicktex.s3tc``, with the same names,
defaults and exceptions. Every encode and decode runs on the GPU through
``libquicktex_cuda.so`` (C-ABI: ``include/quicktex_cuda.h``); there is no CPU
fallback, and importing fails if the native extension was not built
(``python quicktex_b200/build.py``).
"""

import os

from . import _quicktex  # noqa: F401  (native extension; ImportError here means it was not built)
from ._quicktex import RawTexture, Texture, __version__  # noqa: F401

LIBRARY_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libquicktex_cuda.so")


def library_path() -> str:
    """Path of the C-ABI shared library (``include/quicktex_cuda.h``)."""
    return LIBRARY_PATH
