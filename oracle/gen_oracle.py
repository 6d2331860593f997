"""CPU oracle of the learned initialiser's generator (test infrastructure).

A numpy restatement of the network, loss and gradients of
``powerllel_channel_sycl_b200/csrc/plc_gen.cu``, used only by the tests to
check the device kernels: the analytic backward pass here is itself checked
against finite differences in float64, and the device gradients against it.
With ``bf16=True`` the BF16 roundings of the device (weights, convolution
inputs, the gradient operand of the convolutions) are applied at the same
places, so that the remaining differences are FP32 summation order.

Layouts follow the device: tensors [b][z][y][x][c], weights W[tap][co][ci]
with tap = (dz+1)*9 + (dy+1)*3 + (dx+1); convolutions periodic in x and y and
zero-padded in z; FiLM gamma = 1 + A0 + A1 r, beta = B0 + B1 r per (z, c).
"""
from __future__ import annotations

import numpy as np

LEVELS = 4
OUT_C = 16
NSTAT = 31
LAG_BASE = 7


def bf16_round(x):
    """Round to bfloat16 (nearest, ties to even) and back to float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def layer_list(cfg):
    """(ci, co, level, act) of every convolution, in order."""
    ch, lat = cfg["channels"], cfg["latent_channels"]
    out = [(lat, ch[0], 0, True), (ch[0], ch[0], 0, True)]
    for lv in range(1, LEVELS):
        out += [(ch[lv - 1], ch[lv], lv, True), (ch[lv], ch[lv], lv, True)]
    out.append((ch[LEVELS - 1], OUT_C, LEVELS - 1, False))
    return out


def level_dims(cfg, lv):
    sh = LEVELS - 1 - lv
    return cfg["nz"] >> sh, cfg["ny"] >> sh, cfg["nx"] >> sh


def unpack_params(cfg, flat):
    """Views of the flat FP32 parameter vector: [(W, film)] per layer."""
    layers = layer_list(cfg)
    off = 0
    ws = []
    for ci, co, lv, _ in layers:
        n = 27 * co * ci
        ws.append(flat[off:off + n].reshape(27, co, ci))
        off += n
    films = []
    for ci, co, lv, _ in layers:
        z = level_dims(cfg, lv)[0]
        n = 4 * z * co
        films.append(flat[off:off + n].reshape(4, z, co))
        off += n
    assert off == flat.size
    return ws, films


def taps():
    for t in range(27):
        yield t, t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1


def shift(x, dz, dy, dx):
    """x[.., z+dz, y+dy, x+dx, :] (periodic in y, x; zero outside z)."""
    out = np.roll(x, shift=(-dy, -dx), axis=(2, 3))
    if dz == 0:
        return out
    res = np.zeros_like(out)
    if dz > 0:
        res[:, :-dz] = out[:, dz:]
    else:
        res[:, -dz:] = out[:, :dz]
    return res


def conv(x, w):
    y = 0.0
    for t, dz, dy, dx in taps():
        y = y + shift(x, dz, dy, dx) @ w[t].T
    return y


def conv_backward(x, w, dy):
    """(dx, dw) of y = conv(x, w)."""
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    for t, dz, dyy, dxx in taps():
        xs = shift(x, dz, dyy, dxx)
        dw[t] = dy.reshape(-1, dy.shape[-1]).T @ xs.reshape(-1, xs.shape[-1])
        dx += shift(dy @ w[t], -dz, -dyy, -dxx)
    return dx, dw


def upsample(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def upsample_backward(d):
    b, z, y, x, c = d.shape
    return d.reshape(b, z // 2, 2, y // 2, 2, x // 2, 2, c).sum(axis=(2, 4, 6))


def lrelu(h):
    return np.where(h > 0, h, 0.2 * h)


def film_tables(film, r):
    a0, a1, b0, b1 = film
    gam = 1.0 + a0[None] + a1[None] * r[:, None, None]
    bet = b0[None] + b1[None] * r[:, None, None]
    return gam, bet  # [b][z][c]


def forward(cfg, flat, latent, r, bf16=False, dtype=np.float64):
    """Output [b][z][y][x][16] and the saved intermediates."""
    rnd = bf16_round if bf16 else (lambda a: a)
    ws, films = unpack_params(cfg, flat.astype(dtype))
    layers = layer_list(cfg)
    saved = []
    x = rnd(latent.astype(dtype))
    prev_act = None
    for i, (ci, co, lv, act) in enumerate(layers):
        if i > 0 and layers[i - 1][2] != lv:
            x = upsample(prev_act)
        elif i > 0:
            x = prev_act
        w = rnd(ws[i])
        pre = conv(x, w).astype(dtype)
        gam, bet = film_tables(films[i], r.astype(dtype))
        h = gam[:, :, None, None, :] * pre + bet[:, :, None, None, :]
        saved.append((x, w, pre, gam, bet))
        if act:
            prev_act = rnd(lrelu(h))
        else:
            out = h
    return out, saved


def stats(out):
    """Per (b, z) the NSTAT statistics of channels 0-2 (FP64)."""
    f = out[..., :3].astype(np.float64)
    B, Z = f.shape[:2]
    s = np.zeros((B, Z, NSTAT))
    mu = f.mean(axis=(2, 3))
    s[..., 0:3] = mu
    s[..., 3:6] = (f * f).mean(axis=(2, 3)) - mu * mu
    s[..., 6] = (f[..., 0] * f[..., 2]).mean(axis=(2, 3)) - mu[..., 0] * mu[..., 2]
    for c in range(3):
        for q in range(4):
            lag = 1 << q
            sx = (f[..., c] * np.roll(f[..., c], -lag, axis=3)).mean(axis=(2, 3))
            sy = (f[..., c] * np.roll(f[..., c], -lag, axis=2)).mean(axis=(2, 3))
            s[..., LAG_BASE + c * 8 + q] = sx - mu[..., c] ** 2
            s[..., LAG_BASE + c * 8 + 4 + q] = sy - mu[..., c] ** 2
    return s


def loss_and_dout(out, targets, sc_mean, sc_var):
    """Loss against per-sample targets [b][z][NSTAT] and dL/dout."""
    B, Z = out.shape[:2]
    st = stats(out)
    sc = np.full(NSTAT, sc_var)
    sc[:3] = sc_mean
    d = (st - targets) / sc
    norm = 1.0 / (B * Z)
    loss = float((d * d).sum() * norm)
    g = 2.0 * d / sc * norm  # dL/dstat
    f = out[..., :3].astype(np.float64)
    A = f.shape[2] * f.shape[3]
    mu = f.mean(axis=(2, 3))
    dout = np.zeros(out.shape, dtype=np.float64)
    for c in range(3):
        dc = g[..., c][..., None, None] + 2 * g[..., 3 + c][..., None, None] * (f[..., c] - mu[..., c][..., None, None])
        for q in range(4):
            lag = 1 << q
            fc = f[..., c]
            m2 = 2 * mu[..., c][..., None, None]
            dc = dc + g[..., LAG_BASE + c * 8 + q][..., None, None] * (
                np.roll(fc, -lag, axis=3) + np.roll(fc, lag, axis=3) - m2)
            dc = dc + g[..., LAG_BASE + c * 8 + 4 + q][..., None, None] * (
                np.roll(fc, -lag, axis=2) + np.roll(fc, lag, axis=2) - m2)
        dout[..., c] = dc
    dout[..., 0] += g[..., 6][..., None, None] * (f[..., 2] - mu[..., 2][..., None, None])
    dout[..., 2] += g[..., 6][..., None, None] * (f[..., 0] - mu[..., 0][..., None, None])
    return loss, dout / A


def backward(cfg, flat, saved, r, dout, bf16=False):
    """Gradient of every parameter (flat, same layout as the parameters)."""
    rnd = bf16_round if bf16 else (lambda a: a)
    layers = layer_list(cfg)
    grads_w, grads_f = [None] * len(layers), [None] * len(layers)
    d = dout
    for i in range(len(layers) - 1, -1, -1):
        ci, co, lv, act = layers[i]
        x, w, pre, gam, bet = saved[i]
        g4, b4 = gam[:, :, None, None, :], bet[:, :, None, None, :]
        dh = d
        if act:
            h = g4 * pre + b4
            dh = d * np.where(h > 0, 1.0, 0.2)
        dgam = (dh * pre).sum(axis=(2, 3))  # [b][z][c]
        dbet = dh.sum(axis=(2, 3))
        grads_f[i] = np.stack([dgam.sum(0), (dgam * r[:, None, None]).sum(0),
                               dbet.sum(0), (dbet * r[:, None, None]).sum(0)])
        dpre = rnd(dh * g4)
        dx, dw = conv_backward(x, w, dpre)
        grads_w[i] = dw
        if i == 0:
            break
        if layers[i - 1][2] != lv:
            d = upsample_backward(dx)
        else:
            d = dx
    return np.concatenate([g.ravel() for g in grads_w] + [g.ravel() for g in grads_f])


def init_params(cfg, seed=0):
    """He-normal weights (output channels beyond u, v, w zero), zero FiLM."""
    rng = np.random.default_rng(seed)
    parts = []
    for ci, co, lv, act in layer_list(cfg):
        w = rng.normal(0, np.sqrt((2.0 if act else 1.0) / (27 * ci)), (27, co, ci))
        if not act:
            w[:, 3:, :] = 0
        parts.append(w.ravel())
    for ci, co, lv, act in layer_list(cfg):
        parts.append(np.zeros(4 * level_dims(cfg, lv)[0] * co))
    return np.concatenate(parts)
