"""ctypes binding of the warm-start network oracle (oracle/nn_oracle.c).

TEST INFRASTRUCTURE ONLY: the CPU restatement that the GPU network kernels
are checked against.  Arrays are float32 numpy arrays in the layouts of
nn_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnn_oracle.so")
_lib = None

LAYERS = [(8, 16, 1), (16, 16, 1), (16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1),
          (64, 128, 1), (128, 128, 1), (128, 128, 1), (192, 64, 1), (64, 64, 1), (96, 32, 1),
          (32, 32, 1), (48, 16, 1), (16, 16, 1), (16, 4, 0)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        L = C.CDLL(_LIB_PATH)
        vp, i = C.c_void_p, C.c_int
        L.nno_bf16.restype = C.c_float
        L.nno_bf16.argtypes = [C.c_float]
        L.nno_param_count.restype = C.c_longlong
        L.nno_conv_fwd.argtypes = [vp, i, i, i, vp, vp, i, vp, i, i, i, i, i, i]
        L.nno_conv_dgrad.argtypes = [vp, i, i, vp, i, vp, i, i, i, i, i, i]
        L.nno_conv_wgrad.argtypes = [vp, i, i, i, vp, i, i, vp, vp, i, i, i, i]
        L.nno_net.restype = C.c_double
        L.nno_net.argtypes = [vp, i, i, i, i, vp, vp, i, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), kept as float32."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def param_count() -> int:
    return int(lib().nno_param_count())


def conv_fwd(x, cin, w, bias, cout, dims, xs=None, xo=0):
    nb, nz, ny, nx = dims
    m = nb * nz * ny * nx
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros((m, cout), np.float32)
    lib().nno_conv_fwd(_p(x), xs or cin, xo, cin, _p(np.ascontiguousarray(w, np.float32)),
                       _p(None if bias is None else np.ascontiguousarray(bias, np.float32)),
                       cout, _p(y), cout, 0, nb, nz, ny, nx)
    return y


def conv_dgrad(g, cout, w, cin, dims):
    nb, nz, ny, nx = dims
    m = nb * nz * ny * nx
    g = np.ascontiguousarray(g, np.float32)
    dx = np.zeros((m, cin), np.float32)
    lib().nno_conv_dgrad(_p(g), cout, cout, _p(np.ascontiguousarray(w, np.float32)), cin,
                         _p(dx), cin, 0, nb, nz, ny, nx)
    return dx


def conv_wgrad(x, cin, g, cout, dims, xs=None, xo=0):
    nb, nz, ny, nx = dims
    x = np.ascontiguousarray(x, np.float32)
    g = np.ascontiguousarray(g, np.float32)
    dw = np.zeros((cout, 27 * cin), np.float32)
    db = np.zeros(cout, np.float32)
    lib().nno_conv_wgrad(_p(x), xs or cin, xo, cin, _p(g), cout, cout, _p(dw), _p(db),
                         nb, nz, ny, nx)
    return dw, db


def net(params, dims, features, target=None, bf16_mode=True, grads=True):
    """(loss, pred [m, 4], grad or None)."""
    nb, nz, ny, nx = dims
    m = nb * nz * ny * nx
    params = np.ascontiguousarray(params, np.float32)
    feats = np.ascontiguousarray(features, np.float32).reshape(m, 3)
    tgt = None if target is None else np.ascontiguousarray(target, np.float32).reshape(m, 4)
    pred = np.zeros((m, 4), np.float32)
    g = np.zeros_like(params) if (grads and tgt is not None) else None
    loss = lib().nno_net(_p(params), nb, nz, ny, nx, _p(feats), _p(tgt), int(bf16_mode),
                         _p(pred), _p(g))
    return loss, pred, g
