"""Reference counterpart: ``quicktex.s3tc.bc3``."""

from .._quicktex import _s3tc as _s

_m = _s._bc3
__all__ = [n for n in dir(_m) if not n.startswith("_")]
globals().update({n: getattr(_m, n) for n in __all__})
