"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the PES surrogate network
of libqd.so (qd_mlp_*), the checker of its GPU forward and backward kernels.

Same network: features p_ij = exp(-r_ij / 1.5), f = (p23, p12 + p13, p12 p13),
standardised; four dense SiLU layers of width 64; linear output of the
standardised V.  The weights are the GPU's FP32 values (quant=True rounds them
to BF16 first, the arithmetic of an earlier form of the kernels); everything
else is FP64.  Loss: mean squared error
of the standardised V.  Only tests/ load this module.
"""
import numpy as np

W, NF, NL = 64, 3, 4


def layer_off(l):
    return 0 if l == 0 else W * NF + W + (l - 1) * (W * W + W)


OFF_WO = layer_off(NL)
OFF_BO = OFF_WO + W
NPARAM = OFF_BO + 1


def bf16(w):
    """FP32 -> BF16 (nearest even) -> FP64."""
    b = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def _unpack(wq):
    layers = []
    for l in range(NL):
        K = NF if l == 0 else W
        o = layer_off(l)
        layers.append((wq[o:o + W * K].reshape(W, K), wq[o + W * K:o + W * K + W]))
    return layers, wq[OFF_WO:OFF_WO + W], wq[OFF_BO]


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def features(r12, r23, r13, norm):
    p12, p23, p13 = (np.exp(-np.asarray(r, dtype=np.float64) / 1.5) for r in (r12, r23, r13))
    f = np.stack([p23, p12 + p13, p12 * p13], axis=1)
    return (f - norm[0:3].astype(np.float64)) / norm[3:6].astype(np.float64)


def forward(w, norm, r12, r23, r13, quant=False):
    """Standardised output and the per-layer pre-activations and inputs
    (the FP32 weights in FP64 arithmetic; quant=True: rounded to BF16 first)."""
    layers, wo, bo = _unpack(bf16(w) if quant else np.asarray(w, dtype=np.float64))
    a = features(r12, r23, r13, norm)
    zs, ins = [], []
    for Wl, bl in layers:
        ins.append(a)
        z = a @ Wl.T + bl
        zs.append(z)
        a = _silu(z)
    return a @ wo + bo, zs, ins, a


def predict(w, norm, r12, r23, r13):
    """V in hartree."""
    y, *_ = forward(w, norm, r12, r23, r13)
    return y * float(norm[7]) + float(norm[6])


def loss_and_grad(w, norm, r12, r23, r13, V, quant=False):
    """Mean squared error of the standardised V and its gradient with respect
    to the parameters, in the parameter layout of the GPU."""
    layers, wo, bo = _unpack(bf16(w) if quant else np.asarray(w, dtype=np.float64))
    y, zs, ins, a4 = forward(w, norm, r12, r23, r13, quant)
    t = (np.asarray(V, dtype=np.float64) - float(norm[6])) / float(norm[7])
    n = y.size
    e = 2.0 * (y - t) / n
    g = np.zeros(NPARAM)
    g[OFF_WO:OFF_WO + W] = a4.T @ e
    g[OFF_BO] = e.sum()
    d = e[:, None] * wo[None, :] * _dsilu(zs[-1])
    for l in range(NL - 1, -1, -1):
        K = NF if l == 0 else W
        o = layer_off(l)
        g[o:o + W * K] = (d.T @ ins[l]).ravel()
        g[o + W * K:o + W * K + W] = d.sum(axis=0)
        if l > 0:
            d = (d @ layers[l][0]) * _dsilu(zs[l - 1])
    return float(np.mean((y - t) ** 2)), g
