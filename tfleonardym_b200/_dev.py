"""Device plumbing: torch CUDA tensors in, raw pointers and the current stream out."""
import ctypes

import torch

from . import _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("tfleonardym_b200 needs a CUDA device (sm_100a); there is no CPU fallback")


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def as_c128(t, name="tensor"):
    """Return a contiguous complex128 CUDA tensor view/copy of ``t`` (DLPack producers accepted)."""
    if not isinstance(t, torch.Tensor):
        t = torch.from_dlpack(t)
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != torch.complex128:
        t = t.to(torch.complex128)
    return t.contiguous()


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def cdot(a, b):
    """sum conj(a) b as a Python complex (synchronises the current stream)."""
    a = as_c128(a)
    b = as_c128(b)
    if a.shape != b.shape:
        raise RuntimeError("Incompatible vector shapes!")
    out = (ctypes.c_double * 2)()
    _lib.check(_lib.lib().lym_cdot(a.numel(), ptr(a), ptr(b), out, stream()), "lym_cdot")
    return complex(out[0], out[1])


def axpby(a, x, b, y):
    """Return a*x + b*y (complex scalars) as a new tensor, computed by the lym kernel."""
    x = as_c128(x)
    y = as_c128(y)
    if x.shape != y.shape:
        raise RuntimeError("Incompatible vector shapes!")
    out = y.clone()
    ca = (ctypes.c_double * 2)(complex(a).real, complex(a).imag)
    cb = (ctypes.c_double * 2)(complex(b).real, complex(b).imag)
    _lib.check(_lib.lib().lym_caxpby(x.numel(), ca, ptr(x), cb, ptr(out), stream()), "lym_caxpby")
    return out


def axpby_(a, x, b, y):
    """y <- a*x + b*y in place."""
    ca = (ctypes.c_double * 2)(complex(a).real, complex(a).imag)
    cb = (ctypes.c_double * 2)(complex(b).real, complex(b).imag)
    _lib.check(_lib.lib().lym_caxpby(x.numel(), ca, ptr(x), cb, ptr(y), stream()), "lym_caxpby")
    return y
