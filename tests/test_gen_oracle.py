"""The generator's CPU oracle (no GPU): its analytic backward pass against
central finite differences in float64, and the BF16 rounding it emulates."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import gen_oracle as go

CFG = dict(nx=16, ny=16, nz=16, channels=[32, 16, 16, 16], latent_channels=16, batch=2)


def setup(seed=0):
    rng = np.random.default_rng(seed)
    p = go.init_params(CFG, seed=seed)
    # non-trivial FiLM tables so that their gradients are exercised
    nw = sum(27 * ci * co for ci, co, _, _ in go.layer_list(CFG))
    p[nw:] = rng.normal(0, 0.1, p.size - nw)
    lat = rng.normal(size=(CFG["batch"], 2, 2, 2, CFG["latent_channels"]))
    r = np.array([-0.5, 0.7])
    targets = rng.normal(0, 0.05, (CFG["batch"], CFG["nz"], go.NSTAT))
    targets[..., 0] += 1.0
    return p, lat, r, targets


def loss_of(p, lat, r, targets):
    out, _ = go.forward(CFG, p, lat, r)
    return go.loss_and_dout(out, targets, 1.0, 0.05)[0]


def test_param_count_and_layout():
    p = go.init_params(CFG)
    ws, films = go.unpack_params(CFG, p)
    assert len(ws) == 9 and len(films) == 9
    assert ws[-1].shape == (27, 16, 16) and np.all(ws[-1][:, 3:] == 0)
    assert films[0].shape == (4, 2, 32) and films[-1].shape == (4, 16, 16)


def test_backward_matches_finite_differences():
    p, lat, r, targets = setup()
    out, saved = go.forward(CFG, p, lat, r)
    loss, dout = go.loss_and_dout(out, targets, 1.0, 0.05)
    grad = go.backward(CFG, p, saved, r, dout)
    rng = np.random.default_rng(3)
    nw = sum(27 * ci * co for ci, co, _, _ in go.layer_list(CFG))
    # weights of every layer and FiLM parameters (the output rows beyond
    # u, v, w have zero gradient by construction)
    idx = list(rng.choice(nw, 24, replace=False)) + list(nw + rng.choice(p.size - nw, 16, replace=False))
    for i in idx:
        # the LReLU kinks make a large step inexact: take the best of three
        errs = []
        for e in (1e-5, 1e-6, 1e-7):
            pp, pm = p.copy(), p.copy()
            pp[i] += e
            pm[i] -= e
            fd = (loss_of(pp, lat, r, targets) - loss_of(pm, lat, r, targets)) / (2 * e)
            errs.append(abs(fd - grad[i]))
        assert min(errs) <= 1e-6 * max(1.0, abs(grad[i])), (i, grad[i], errs)


def test_stats_definitions():
    rng = np.random.default_rng(1)
    out = rng.normal(size=(1, 3, 8, 8, 16))
    s = go.stats(out)
    f = out[0, 1, :, :, 0]
    assert np.isclose(s[0, 1, 0], f.mean())
    assert np.isclose(s[0, 1, 3], f.var())
    lag2x = ((f - f.mean()) * (np.roll(f, -2, axis=1) - f.mean())).mean()
    assert np.isclose(s[0, 1, go.LAG_BASE + 1], lag2x)
    lag4y = ((f - f.mean()) * (np.roll(f, -4, axis=0) - f.mean())).mean()
    assert np.isclose(s[0, 1, go.LAG_BASE + 4 + 2], lag4y)


def test_bf16_round():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 1e-30, 65504.0], np.float32)
    y = go.bf16_round(x)
    assert y[0] == 1.0
    assert y[1] == 1.0  # halfway between 1 and 1 + 2^-7: ties to even
    assert y[2] == np.float32(1.0078125)
    assert abs(y[3] + 3.140625) < 1e-7
    assert np.all(np.abs(y - x) <= np.abs(x) * 2 ** -8)
