"""S3TC encoders and decoders (reference: ``quicktex.s3tc``)."""

from . import bc1, bc3, bc4, bc5, interpolator  # noqa: F401
