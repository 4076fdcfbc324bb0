"""dot (mirror of algebra_utils.py:5-11), computed by the lym reduction kernel."""
from . import _dev


def dot(v1, v2):
    if tuple(v1.shape) != tuple(v2.shape):
        raise RuntimeError("Incompatible vector shapes!")
    return _dev.cdot(v1, v2)
