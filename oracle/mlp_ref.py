"""CPU oracle of the learned-guess network (test infrastructure only; the product never imports it).

A plain numpy restatement of what the library's MLP kernels compute, used to check them:
  forward   z_l = bf16(x_l) bf16(W_l)^T + b_l,  x_{l+1} = silu(z_l) (hidden layers), y = z_{L-1}
  loss      sum(mask (y - t)^2) / sum(mask)
  backward  dW_l = bf16(dz_l)^T bf16(x_l),  db_l = sum_rows dz_l,  dx_l = bf16(dz_l) bf16(W_l),
            dz_l = dx_{l+1} silu'(z_l) for hidden layers
with every matrix-product operand rounded to BF16 (round to nearest even) and FP32 accumulation, and the
parameter layout of include/qchem_b200.h (per layer W (out x in) then b (out)).  The reference qchem has
no learned component; this oracle is pinned by a finite-difference check of its own gradient.
"""
import numpy as np


def bf16(x):
    """Round float32 values to the nearest BF16 value (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def unpack(params, widths):
    Ws, bs, off = [], [], 0
    for l in range(len(widths) - 1):
        i, o = widths[l], widths[l + 1]
        Ws.append(params[off:off + o * i].reshape(o, i))
        off += o * i
        bs.append(params[off:off + o])
        off += o
    return Ws, bs


def nparams(widths):
    return sum(widths[l + 1] * widths[l] + widths[l + 1] for l in range(len(widths) - 1))


def _silu(z):
    return z / (1.0 + np.exp(-z))


def forward(params, widths, x, keep=False, round_bf16=True, dtype=np.float32):
    """round_bf16=False with dtype=np.float64 gives the exact-arithmetic network (for the gradient pin)."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=dtype))
    Ws, bs = unpack(np.asarray(params, dtype=dtype), widths)
    xs, zs = [np.asarray(x, dtype=dtype)], []
    L = len(Ws)
    for l in range(L):
        z = (r(xs[-1]) @ r(Ws[l]).T + bs[l]).astype(dtype)
        zs.append(z)
        xs.append(_silu(z).astype(dtype) if l + 1 < L else z)
    return (xs, zs) if keep else xs[-1]


def loss_grad(params, widths, x, t, mask, round_bf16=True, dtype=np.float32):
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=dtype))
    Ws, _ = unpack(np.asarray(params, dtype=dtype), widths)
    xs, zs = forward(params, widths, x, keep=True, round_bf16=round_bf16, dtype=dtype)
    y = xs[-1]
    msum = float(mask.sum())
    res = mask * (y - t)
    loss = float((res.astype(np.float64) ** 2).sum() / msum)
    d = (2.0 * res / msum).astype(dtype)
    grads = []
    L = len(Ws)
    for l in range(L - 1, -1, -1):
        if l + 1 < L:
            s = 1.0 / (1.0 + np.exp(-zs[l]))
            d = (d * s * (1.0 + zs[l] * (1.0 - s))).astype(dtype)
        gW = (r(d).T @ r(xs[l])).astype(dtype)
        gb = d.sum(axis=0).astype(dtype)
        grads.append((gW, gb))
        if l > 0:
            d = (r(d) @ r(Ws[l])).astype(dtype)
    g = []
    for gW, gb in reversed(grads):
        g.append(gW.ravel())
        g.append(gb)
    return loss, np.concatenate(g)
