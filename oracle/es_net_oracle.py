"""CPU FP64 restatement of the learned early-stop network (test infrastructure
only: the product path is the CUDA network in special-topics_b200/csrc/es_net.cu).

Same architecture, parameter layout and loss as the C ABI documents
(include/fdtd_b200.h, fdtd_es_*): convolutions with zero padding kernel//2 and
ReLU over time-major, channel-fastest samples; dense layers with ReLU; a
linear head; L = mean_b sum_o w[o] (y - t)^2.  With bf16=True the weights enter
the arithmetic as their BF16 values (round to nearest even of the FP32
master) and the biases as FP32, as on the GPU; everything else is FP64.  The
analytic backward pass is the reference the GPU gradients are checked
against; with bf16=False it is the exact derivative of `loss`, which
`finite_difference` checks.
"""
from __future__ import annotations

import numpy as np

DEFAULT_ARCH = dict(in_channels=2, in_length=375, conv_layers=4, channels=64, kernel=5, stride=2,
                    mlp_layers=2, mlp_width=256)


def bf16_round(a) -> np.ndarray:
    """FP32 -> nearest BF16 (ties to even), returned as FP32."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    nan = ((x & 0x7F800000) == 0x7F800000) & ((x & 0x007FFFFF) != 0)
    lsb = (x >> 16) & 1
    r = (x + 0x7FFF + lsb) & 0xFFFF0000
    r = np.where(nan, (x | 0x00400000) & 0xFFFF0000, r)   # NaNs stay (quiet) NaNs
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(a))


def layers(arch: dict, out_dim: int) -> list[dict]:
    """Layer list with (offset, shape) of each weight and bias, in the flat order of the C ABI."""
    out, off = [], 0
    length, ch = arch["in_length"], arch["in_channels"]
    K, S = arch["kernel"], arch["stride"]
    for _ in range(arch["conv_layers"]):
        pad = K // 2
        lout = (length + 2 * pad - K) // S + 1
        L = dict(conv=True, cin=ch, cout=arch["channels"], lin=length, lout=lout, k=K, s=S, pad=pad, relu=True,
                 w=(off, (arch["channels"], K, ch)))
        off += arch["channels"] * K * ch
        L["b"] = (off, (arch["channels"],))
        off += arch["channels"]
        out.append(L)
        length, ch = lout, arch["channels"]
    feat = length * ch
    for q in range(arch["mlp_layers"] + 1):
        cout = arch["mlp_width"] if q < arch["mlp_layers"] else out_dim
        L = dict(conv=False, cin=feat, cout=cout, relu=q < arch["mlp_layers"], w=(off, (cout, feat)))
        off += cout * feat
        L["b"] = (off, (cout,))
        off += cout
        out.append(L)
        feat = cout
    return out


def param_count(arch: dict, out_dim: int) -> int:
    L = layers(arch, out_dim)[-1]
    return L["b"][0] + L["b"][1][0]


def _weights(params, L, bf16: bool):
    off, shape = L["w"]
    W = np.asarray(params[off:off + int(np.prod(shape))]).reshape(shape)
    W = bf16_round(W).astype(np.float64) if bf16 else np.asarray(W, dtype=np.float64)
    off, shape = L["b"]
    b = np.asarray(params[off:off + shape[0]])
    b = b.astype(np.float32).astype(np.float64) if bf16 else np.asarray(b, dtype=np.float64)
    return W, b


def _im2col(x, L):
    """x: (B, lin, cin) -> (B, lout, k, cin), zero outside [0, lin)."""
    B = x.shape[0]
    xp = np.zeros((B, L["lin"] + 2 * L["pad"] + L["k"], L["cin"]))
    xp[:, L["pad"]:L["pad"] + L["lin"]] = x
    idx = np.arange(L["lout"])[:, None] * L["s"] + np.arange(L["k"])[None, :]
    return xp[:, idx, :]


def forward(arch: dict, out_dim: int, params, x, bf16: bool = True):
    """x: (B, in_length, in_channels).  Returns y (B, out_dim) and the cache."""
    a = np.asarray(x, dtype=np.float64)
    cache = []
    for L in layers(arch, out_dim):
        W, b = _weights(params, L, bf16)
        if L["conv"]:
            cols = _im2col(a, L)
            z = np.einsum("btkc,okc->bto", cols, W) + b
        else:
            cols = a.reshape(a.shape[0], -1)
            z = cols @ W.T + b
        out = np.maximum(z, 0.0) if L["relu"] else z
        cache.append((L, a.shape, cols, out, W))
        a = out
    return a, cache


def loss(arch: dict, out_dim: int, params, x, target, w, bf16: bool = True) -> float:
    y, _ = forward(arch, out_dim, params, x, bf16)
    r = y - np.asarray(target, dtype=np.float64)
    return float(np.sum(np.asarray(w, dtype=np.float64) * r * r) / y.shape[0])


def loss_grad(arch: dict, out_dim: int, params, x, target, w, bf16: bool = True):
    """Loss and its gradient with respect to the flat parameter vector."""
    y, cache = forward(arch, out_dim, params, x, bf16)
    B = y.shape[0]
    r = y - np.asarray(target, dtype=np.float64)
    w = np.asarray(w, dtype=np.float64)
    value = float(np.sum(w * r * r) / B)
    d = 2.0 * w * r / B
    grad = np.zeros(len(params))
    for L, in_shape, cols, out, W in reversed(cache):
        if L["relu"]:
            d = d * (out > 0)
        off_w, _ = L["w"]
        off_b, _ = L["b"]
        if L["conv"]:
            gW = np.einsum("bto,btkc->okc", d, cols)
            grad[off_b:off_b + L["cout"]] = d.sum(axis=(0, 1))
            dcols = np.einsum("bto,okc->btkc", d, W)
            dx = np.zeros((in_shape[0], L["lin"] + 2 * L["pad"] + L["k"], L["cin"]))
            for k in range(L["k"]):
                dx[:, k:k + L["s"] * L["lout"]:L["s"], :] += dcols[:, :, k, :]
            d = dx[:, L["pad"]:L["pad"] + L["lin"], :]
        else:
            gW = d.T @ cols
            grad[off_b:off_b + L["cout"]] = d.sum(axis=0)
            d = (d @ W).reshape(in_shape)
        grad[off_w:off_w + gW.size] = gW.ravel()
    return value, grad


def finite_difference(arch: dict, out_dim: int, params, x, target, w, idx, h: float = 1e-5) -> np.ndarray:
    """Central differences of `loss` (bf16=False) at the listed parameter indices."""
    p = np.asarray(params, dtype=np.float64)
    out = []
    for q in idx:
        p1, p2 = p.copy(), p.copy()
        p1[q] += h
        p2[q] -= h
        out.append((loss(arch, out_dim, p1, x, target, w, False) - loss(arch, out_dim, p2, x, target, w, False))
                   / (2 * h))
    return np.array(out)
