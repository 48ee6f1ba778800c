"""TEST INFRASTRUCTURE ONLY (oracle): FP64 numpy forward / backward of the
surrogate MLP, for checking the device kernels' gradients.  The MLP has no
counterpart in the reference; this restates the network the library trains
(bnm_cuda_b200/csrc/mlp.cu) with the same rounding points:

  forward   Z_l = bf16(A_l) bf16(W_l)^T + b_l ; A_{l+1} = bf16(relu(Z_l)) for
            hidden layers, the last layer's Z kept in float;
  loss      mean over batch and outputs of (Y - T)^2;
  backward  dY = 2 (Y - T) / (B O); for each layer dZ = dY * 1[A_{l+1} > 0]
            (hidden); db = sum_b dZ (unrounded); dW = bf16(dZ)^T A_l;
            dX = bf16(dZ) bf16(W_l).

Parameters are flat, per layer W [out][in] then b [out].
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (round to nearest even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    rounding = 0x7FFF + ((b >> 16) & 1)
    b = ((b + rounding) & 0xFFFF0000).astype(np.uint32)
    out = b.view(np.float32).astype(np.float64)
    nan = np.isnan(f)
    out[nan] = np.nan
    return out


def unflatten(flat: np.ndarray, dims):
    Ws, bs, off = [], [], 0
    for din, dout in zip(dims[:-1], dims[1:]):
        Ws.append(flat[off:off + din * dout].astype(np.float64).reshape(dout, din))
        off += din * dout
        bs.append(flat[off:off + dout].astype(np.float64))
        off += dout
    return Ws, bs


def loss_and_grads(flat: np.ndarray, dims, X: np.ndarray, T: np.ndarray):
    Ws, bs = unflatten(flat, dims)
    L = len(Ws)
    acts = [bf16(X)]
    Y = None
    for l in range(L):
        Z = acts[l] @ bf16(Ws[l]).T + bs[l]
        if l < L - 1:
            acts.append(bf16(np.maximum(Z, 0.0)))
        else:
            Y = Z.astype(np.float32).astype(np.float64)
    B, O = Y.shape
    diff = Y - T
    loss = float(np.mean(diff ** 2))
    dY = (2.0 * diff / (B * O)).astype(np.float32).astype(np.float64)
    grads = []
    for l in range(L - 1, -1, -1):
        dZ = dY if l == L - 1 else dY * (acts[l + 1] > 0)
        db = dZ.sum(0)
        dW = bf16(dZ).T @ acts[l]
        grads.append((dW, db))
        if l > 0:
            dY = (bf16(dZ) @ bf16(Ws[l])).astype(np.float32).astype(np.float64)
    flat_g = []
    for dW, db in reversed(grads):
        flat_g.append(dW.ravel())
        flat_g.append(db)
    return loss, np.concatenate(flat_g), Y
