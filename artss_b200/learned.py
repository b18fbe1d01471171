"""Learned initial guess of the pressure solve: a small 3-D U-Net whose
convolutions run on the tensor cores (include/artss_cuda.h, artss_conv3d_*).
No counterpart in the reference.

Host-side helpers: BF16 conversion and the weight packing the convolution
kernels expect.  Device buffers are torch tensors used as plain memory; every
operation on them is a kernel of libartss_cuda.so."""
from __future__ import annotations

import numpy as np


def to_bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.ascontiguousarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def round_bf16(a: np.ndarray) -> np.ndarray:
    return from_bf16_bits(to_bf16_bits(a))


def pack_conv_weights(w: np.ndarray) -> np.ndarray:
    """w[co][ci][kz][ky][kx] -> [27][ci/8][co][8] (tap t = 9 kz + 3 ky + kx),
    the per-tap shared-memory layout of the convolution's B operand."""
    co, ci = w.shape[:2]
    assert w.shape[2:] == (3, 3, 3) and ci % 8 == 0
    t = np.ascontiguousarray(w.reshape(co, ci, 27).transpose(2, 1, 0))  # [27][ci][co]
    return np.ascontiguousarray(t.reshape(27, ci // 8, 8, co).transpose(0, 1, 3, 2))  # [27][ci/8][co][8]


def conv3d_ref(x: np.ndarray, w: np.ndarray, bias=None, relu=False) -> np.ndarray:
    """FP32 reference: x[D][H][W][ci], w[co][ci][3][3][3], zero padding 1."""
    D, H, W, ci = x.shape
    co = w.shape[0]
    xp = np.zeros((D + 2, H + 2, W + 2, ci), np.float32)
    xp[1:-1, 1:-1, 1:-1] = x
    y = np.zeros((D, H, W, co), np.float32)
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                y += np.einsum("zyxc,oc->zyxo", xp[kz:kz + D, ky:ky + H, kx:kx + W], w[:, :, kz, ky, kx],
                               optimize=True)
    if bias is not None:
        y += bias
    if relu:
        y = np.maximum(y, 0)
    return y


def flip_weights(w: np.ndarray) -> np.ndarray:
    """Weights of the input-gradient convolution: w'[ci][co][t] = w[co][ci][26 - t]."""
    return np.ascontiguousarray(w.transpose(1, 0, 2, 3, 4)[:, :, ::-1, ::-1, ::-1])


def conv3d_wgrad_ref(x: np.ndarray, dy: np.ndarray) -> np.ndarray:
    """FP32 reference: dw[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci]."""
    D, H, W, ci = x.shape
    co = dy.shape[3]
    xp = np.zeros((D + 2, H + 2, W + 2, ci), np.float32)
    xp[1:-1, 1:-1, 1:-1] = x
    dw = np.zeros((27, co, ci), np.float32)
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                dw[9 * kz + 3 * ky + kx] = np.einsum("zyxo,zyxc->oc", dy, xp[kz:kz + D, ky:ky + H, kx:kx + W],
                                                     optimize=True)
    return dw
