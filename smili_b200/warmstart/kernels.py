"""ctypes binding of ``libsmili_unet.so`` (declared in include/smili_unet.h).

Every function takes torch CUDA tensors (or None), passes their device
pointers, launches on torch's current stream and raises on a nonzero status.
There is no fallback: the library must be built (``smili_b200.build``).
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(HERE, "libsmili_unet.so")

EXPORTS = ["smili_unet_conv3x3", "smili_unet_conv3x3_wgrad", "smili_unet_bias_grad", "smili_unet_flip_weights",
           "smili_unet_relu_mask", "smili_unet_avgpool2", "smili_unet_avgpool2_bwd", "smili_unet_upsample2",
           "smili_unet_upsample2_bwd", "smili_unet_mse", "smili_unet_adam", "smili_unet_f32_to_bf16",
           "smili_unet_set_conv_path", "smili_unet_tc_status", "smili_unet_last_error"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with smili_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        vp, i, ll, f = C.c_void_p, C.c_int, C.c_longlong, C.c_float
        sig = {
            "smili_unet_conv3x3": [vp, i, i, i, i, i, vp, vp, vp, i, i, i, i, vp],
            "smili_unet_conv3x3_wgrad": [vp, i, vp, i, i, i, i, i, i, vp, i, vp, i, vp],
            "smili_unet_bias_grad": [vp, i, ll, i, vp, i, vp],
            "smili_unet_flip_weights": [vp, vp, i, i, vp],
            "smili_unet_relu_mask": [vp, i, vp, i, ll, i, vp],
            "smili_unet_avgpool2": [vp, i, vp, i, i, i, i, i, vp],
            "smili_unet_avgpool2_bwd": [vp, i, vp, i, i, i, i, i, i, vp],
            "smili_unet_upsample2": [vp, i, vp, i, i, i, i, i, vp],
            "smili_unet_upsample2_bwd": [vp, i, vp, i, i, i, i, i, i, vp],
            "smili_unet_mse": [vp, i, vp, ll, vp, i, vp, i, vp],
            "smili_unet_adam": [vp, vp, vp, vp, vp, ll, f, f, f, f, f, i, vp],
            "smili_unet_f32_to_bf16": [vp, vp, ll, vp],
            "smili_unet_set_conv_path": [i],
            "smili_unet_tc_status": [],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.smili_unet_last_error.argtypes = []
        L.smili_unet_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def _p(t):
    """Device pointer of a tensor (or a (tensor, element offset) slice), or None."""
    if t is None:
        return None
    if isinstance(t, tuple):
        base, off = t
        return base.data_ptr() + off * base.element_size()
    return t.data_ptr()


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _check(rc, name):
    if rc != 0:
        why = (lib().smili_unet_last_error() or b"").decode()
        raise RuntimeError(f"{name} failed with status {rc}" + (f": {why}" if why else ""))


def conv3x3(x, N, H, W, Cin, ldx, w, bias, y, ldy, Cout, relu, accumulate=False):
    _check(lib().smili_unet_conv3x3(_p(x), N, H, W, Cin, ldx, _p(w), _p(bias), _p(y), ldy, Cout, int(relu),
                                    int(accumulate), _stream()), "conv3x3")


def conv3x3_wgrad(x, ldx, dy, lddy, N, H, W, Cin, Cout, partial, nsplit, dw, accumulate=False):
    _check(lib().smili_unet_conv3x3_wgrad(_p(x), ldx, _p(dy), lddy, N, H, W, Cin, Cout, _p(partial), nsplit,
                                          _p(dw), int(accumulate), _stream()), "conv3x3_wgrad")


def bias_grad(dy, ld, npix, C_, db, accumulate=False):
    _check(lib().smili_unet_bias_grad(_p(dy), ld, npix, C_, _p(db), int(accumulate), _stream()), "bias_grad")


def flip_weights(w, wt, Cout, Cin):
    _check(lib().smili_unet_flip_weights(_p(w), _p(wt), Cout, Cin, _stream()), "flip_weights")


def relu_mask(y, ldy, dy, lddy, npix, C_):
    _check(lib().smili_unet_relu_mask(_p(y), ldy, _p(dy), lddy, npix, C_, _stream()), "relu_mask")


def avgpool2(x, ldx, y, ldy, N, H, W, C_):
    _check(lib().smili_unet_avgpool2(_p(x), ldx, _p(y), ldy, N, H, W, C_, _stream()), "avgpool2")


def avgpool2_bwd(dy, lddy, dx, lddx, N, H, W, C_, accumulate=False):
    _check(lib().smili_unet_avgpool2_bwd(_p(dy), lddy, _p(dx), lddx, N, H, W, C_, int(accumulate), _stream()),
           "avgpool2_bwd")


def upsample2(x, ldx, y, ldy, N, H, W, C_):
    _check(lib().smili_unet_upsample2(_p(x), ldx, _p(y), ldy, N, H, W, C_, _stream()), "upsample2")


def upsample2_bwd(dy, lddy, dx, lddx, N, H, W, C_, accumulate=False):
    _check(lib().smili_unet_upsample2_bwd(_p(dy), lddy, _p(dx), lddx, N, H, W, C_, int(accumulate), _stream()),
           "upsample2_bwd")


def mse(y, ldy, target, n, dy, lddy, loss_part, nblocks):
    _check(lib().smili_unet_mse(_p(y), ldy, _p(target), n, _p(dy), lddy, _p(loss_part), nblocks, _stream()), "mse")


def adam(w, w16, g, m, v, n, lr, b1, b2, eps, wd, step):
    _check(lib().smili_unet_adam(_p(w), _p(w16), _p(g), _p(m), _p(v), n, lr, b1, b2, eps, wd, step, _stream()),
           "adam")


def f32_to_bf16(x, y, n):
    _check(lib().smili_unet_f32_to_bf16(_p(x), _p(y), n, _stream()), "f32_to_bf16")


def set_conv_path(path):
    """0: tcgen05 convolutions where they apply (default); 1: mma.sync always."""
    _check(lib().smili_unet_set_conv_path(int(path)), "set_conv_path")


def tc_status():
    """Read and clear the tcgen05 convolution's error flag (0: no bounded wait ran out)."""
    return int(lib().smili_unet_tc_status())
