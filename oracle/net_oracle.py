"""CPU FP32 oracle of the proposal network (TEST INFRASTRUCTURE ONLY).

numpy restatement of the forward pass, loss and backward pass that
librcmvs's tensor-core kernels implement (rcmvs_net_train_step), used by the
tests to check the GPU gradients.  With bf16=True it rounds the tensors the
GPU stores in BF16 (input, weights, hidden activations, loss gradient,
back-propagated gradients) at the same points, so the comparison isolates
the accumulation order.  The network has no counterpart in the reference.
"""
import numpy as np

CIN = [48, 32, 32, 32, 32, 32]
CIN_REAL = [33, 32, 32, 32, 32, 32]
COUT = [32, 32, 32, 32, 32, 16]
COUT_REAL = [32, 32, 32, 32, 32, 5]
LN, LC = 1.0, 0.1


def param_layout():
    out, off = [], 0
    for ci, co in zip(CIN, COUT):
        w = (off, 9 * co * ci)
        off += 9 * co * ci
        b = (off, co)
        off += co
        out.append((w, b, ci, co))
    return out, off


def unpack(params):
    lay, _ = param_layout()
    Ws, bs = [], []
    for (wo, wn), (bo, bn), ci, co in lay:
        Ws.append(params[wo:wo + wn].reshape(9, co, ci))
        bs.append(params[bo:bo + bn])
    return Ws, bs


def pack(Ws, bs):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in zip(Ws, bs)]).astype(np.float32)


def bf16(a):
    """Round float32 to the nearest bfloat16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


def _patches(x):
    """x (N,H,W,C) -> (N,H,W,9,C): the 3x3 neighbourhood, zero padded, tap = ky*3+kx."""
    n, h, w, c = x.shape
    xp = np.zeros((n, h + 2, w + 2, c), x.dtype)
    xp[:, 1:-1, 1:-1] = x
    return np.stack([xp[:, ky:ky + h, kx:kx + w] for ky in range(3) for kx in range(3)], axis=3)


def conv(x, W, b):
    """y[n,y,x,co] = b[co] + sum_{tap,ci} W[tap,co,ci] x[n,y+ky-1,x+kx-1,ci]."""
    y = np.einsum("nhwtc,toc->nhwo", _patches(x), W, optimize=True).astype(np.float32)
    return y + (b if b is not None else 0)


def conv_back_data(dy, W):
    """Gradient of conv wrt its input: the transposed convolution."""
    # dx[p][ci] = sum_{t, co} W[t][co][ci] dy[p - off(t)][co] and -off(t) = off(8 - t)
    return np.einsum("nhwto,toc->nhwc", _patches(dy), W[::-1], optimize=True).astype(np.float32)


def conv_back_weights(x, dy):
    return np.einsum("nhwtc,nhwo->toc", _patches(x), dy, optimize=True).astype(np.float32)


def loss_and_grad(out, lab):
    """out (..,16) f32, lab (..,8) -> (mean loss over valid, dL/dout unscaled, count)."""
    valid = lab[..., 4] > 0.5
    g = np.zeros_like(out)
    t, ts = out[..., 0], lab[..., 0]
    dt = t - ts
    nvec = out[..., 1:4]
    nl = np.sqrt((nvec ** 2).sum(-1)) + 1e-6
    c = (nvec * lab[..., 1:4]).sum(-1) / nl
    pr = 1.0 / (1.0 + np.exp(-out[..., 4]))
    tgt = (np.abs(dt) < lab[..., 5]).astype(np.float32)
    l = np.abs(dt) + LN * (1 - c) - LC * (tgt * np.log(np.maximum(pr, 1e-7)) +
                                          (1 - tgt) * np.log(np.maximum(1 - pr, 1e-7)))
    g[..., 0] = np.sign(dt)
    g[..., 1:4] = -LN * (lab[..., 1:4] - c[..., None] * nvec / nl[..., None]) / nl[..., None]
    g[..., 4] = LC * (pr - tgt)
    g[~valid] = 0
    n = max(int(valid.sum()), 1)
    return float(l[valid].sum() / n), g, n


def forward(params, x, bf=True):
    Ws, bs = unpack(np.asarray(params, np.float32))
    r = bf16 if bf else (lambda a: a)
    Ws = [r(w) for w in Ws]
    acts = [r(x)]
    for l in range(6):
        y = conv(acts[-1], Ws[l], bs[l])
        if l < 5:
            acts.append(r(np.maximum(y, 0)))
        else:
            acts.append(y.astype(np.float32))
    return acts, Ws, bs


def gradients(params, x, lab, bf=True):
    """Mean loss and its gradient wrt the parameters (parameter layout)."""
    r = bf16 if bf else (lambda a: a)
    acts, Ws, bs = forward(params, x, bf)
    loss, g, n = loss_and_grad(acts[-1], lab)
    dy = r(g)
    dWs, dbs = [None] * 6, [None] * 6
    for l in range(5, -1, -1):
        dpre = dy if l == 5 else dy * (acts[l + 1] > 0)
        dWs[l] = conv_back_weights(acts[l], dpre) / n
        dbs[l] = dpre.sum(axis=(0, 1, 2)) / n
        if l > 0:
            dy = r(conv_back_data(dpre, Ws[l]))
    lay, _ = param_layout()
    for l in range(6):  # padded entries carry no gradient on the GPU either way
        dWs[l][:, COUT_REAL[l]:, :] = 0
        dWs[l][:, :, CIN_REAL[l]:] = 0
        dbs[l][COUT_REAL[l]:] = 0
    return loss, pack(dWs, dbs)
