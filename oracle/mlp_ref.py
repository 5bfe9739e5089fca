"""FP64 CPU oracle of the surrogate MLP (test infrastructure only).

Same architecture and parameter layout as dg_mlp (include/diskgpu.h): per layer W
(fan_out x fan_in) then b; SiLU hidden layers, linear head, mean-squared-error loss.
The weights are rounded to BF16 first, as the GPU kernels use them, so the comparison
isolates the FP32-vs-FP64 arithmetic.  Gradients are w.r.t. the master weights.
"""
import numpy as np


def bf16_round(x):
    """Round FP32 values to the nearest BF16 (ties to even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(params, n_in, width, depth, n_out):
    out, off = [], 0
    fin = n_in
    for l in range(depth + 1):
        fo = n_out if l == depth else width
        W = params[off: off + fo * fin].reshape(fo, fin)
        off += fo * fin
        b = params[off: off + fo]
        off += fo
        out.append((W, b))
        fin = fo
    return out


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(params, x, n_in, width, depth, n_out, round_bf16=True):
    Ls = layers(np.asarray(params, dtype=np.float64), n_in, width, depth, n_out)
    a = np.asarray(x, dtype=np.float64)
    for l, (W, b) in enumerate(Ls):
        Wc = bf16_round(W) if round_bf16 else W
        z = a @ Wc.T + b
        a = _silu(z) if l < depth else z
    return a


def loss_grad(params, x, t, n_in, width, depth, n_out, round_bf16=True):
    P = np.asarray(params, dtype=np.float64)
    Ls = layers(P, n_in, width, depth, n_out)
    acts, zs = [np.asarray(x, dtype=np.float64)], []
    for l, (W, b) in enumerate(Ls):
        Wc = bf16_round(W) if round_bf16 else W
        z = acts[-1] @ Wc.T + b
        zs.append(z)
        acts.append(_silu(z) if l < depth else z)
    y = acts[-1]
    d = y - np.asarray(t, dtype=np.float64)
    loss = float(np.mean(d * d))
    dout = 2.0 * d / d.size
    grads = []
    for l in range(depth, -1, -1):
        W, b = Ls[l]
        Wc = bf16_round(W) if round_bf16 else W
        grads.append((dout.T @ acts[l], dout.sum(axis=0)))
        if l > 0:
            dout = (dout @ Wc) * _silu_grad(zs[l - 1])
    flat = []
    for dW, db in reversed(grads):
        flat += [dW.ravel(), db]
    return loss, np.concatenate(flat)
