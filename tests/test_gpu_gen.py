"""The generator's device kernels against the CPU oracle (BF16 roundings
emulated at the same places): forward output, statistics, loss and every
parameter gradient; training, the coarse-grained snapshot statistics, the
projection and the proposal into a channel."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import case_kwargs, channel_params, interior
from oracle import gen_oracle as go

pytestmark = pytest.mark.gpu

SMALL = dict(nx=16, ny=16, nz=16, channels=[32, 16, 16, 16], latent_channels=16, batch=2)


def make_gen(**over):
    from powerllel_channel_sycl_b200.learned import Generator, config
    kw = dict(SMALL, **over)
    return Generator(config(**kw, seed=5)), kw


def rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def test_forward_matches_oracle():
    g, cfg = make_gen()
    re = np.array([180.0, 395.0])
    out = g.forward(re, seed=11)
    lat = g.latent(11)
    p = g.params.astype(np.float64)
    ref, _ = go.forward(cfg, p, lat, (re - 260) / 140, bf16=True)
    assert out.shape == (2, 16, 16, 16, 3)
    assert rel(out, ref[..., :3]) < 2e-3
    st = g.output_stats()
    full = np.concatenate([out, np.zeros(out.shape[:-1] + (13,), np.float32)], -1)
    assert rel(st, go.stats(full)) < 1e-5


def test_loss_and_gradients_match_oracle():
    g, cfg = make_gen()
    rng = np.random.default_rng(2)
    targets = rng.normal(0, 0.02, (3, 16, go.NSTAT))
    targets[..., 0] += np.linspace(0.2, 1.0, 16)
    targets[..., 3:6] += 0.01
    re_t = np.array([150.0, 250.0, 380.0])
    g.set_targets(re_t, targets)
    tidx = np.array([2, 0], np.int32)
    loss, grad = g.loss_grad(tidx, re_t[tidx], seed=7)
    lat = g.latent(7)
    p = g.params.astype(np.float64)
    r = (re_t[tidx] - 260) / 140
    out, saved = go.forward(cfg, p, lat, r, bf16=True)
    sc_mean = np.sqrt(np.mean(targets[..., 0] ** 2))
    sc_var = np.sqrt(np.mean(targets[..., 3] ** 2))
    lref, dout = go.loss_and_dout(out, targets[tidx], sc_mean, sc_var)
    gref = go.backward(cfg, p, saved, r, dout, bf16=True)
    assert abs(loss - lref) <= 1e-4 * lref
    assert rel(grad, gref) < 2e-2
    # per layer too: every layer's weight gradient and the FiLM gradients
    off = 0
    for ci, co, lv, act in go.layer_list(cfg):
        n = 27 * ci * co
        sl = slice(off, off + n)
        if np.linalg.norm(gref[sl]) > 0:
            assert rel(grad[sl], gref[sl]) < 5e-2, (ci, co, lv)
        off += n
    assert rel(grad[off:], gref[off:]) < 2e-2


def test_training_reduces_loss():
    g, cfg = make_gen(batch=4)
    # targets: statistics of smooth random fields with a mean profile
    rng = np.random.default_rng(0)
    tg = []
    for q in range(4):
        f = rng.normal(size=(1, 16, 16, 16, 16)) * 0.1
        f = (f + np.roll(f, 1, 3) + np.roll(f, 1, 2)) / 3
        z = (np.arange(16) + 0.5) / 16
        f[..., 0] += (1 - (2 * z - 1) ** 2)[None, :, None, None] * (0.8 + 0.1 * q)
        tg.append(go.stats(f)[0])
    g.set_targets(np.array([150.0, 220.0, 300.0, 390.0]), np.array(tg))
    hist = g.train(300, lr=3e-3, seed=3)
    assert np.all(np.isfinite(hist))
    assert hist[-20:].mean() < 0.2 * hist[:20].mean(), (hist[:5], hist[-5:])


def _channel(nx, ny, nz, precision=0):
    from powerllel_channel_sycl_b200 import Channel
    prm = channel_params(**case_kwargs(nx, ny, nz))
    prm.precision = precision
    return Channel(prm)


@pytest.mark.parametrize("precision", [0, 1])
def test_projection_makes_fields_divergence_free(precision):
    ch = _channel(32, 24, 16, precision)
    rng = np.random.default_rng(4)
    for q in "uvw":
        ch.upload(q, rng.normal(size=ch.shape))
    ch.project()
    div = ch.check()[2][0]
    assert div < (1e-12 if precision == 0 else 1e-4), div


def test_stats_of_channel_matches_numpy():
    g, _ = make_gen()
    ch = _channel(32, 32, 32)
    ch.initFlow()
    ch.step(3)
    st = g.stats_of(ch)
    u, v, w = (ch.download(q) for q in "uvw")
    uc = 0.5 * (u[1:-1, 1:-1, 1:-1] + u[1:-1, 1:-1, :-2])
    vc = 0.5 * (v[1:-1, 1:-1, 1:-1] + v[1:-1, :-2, 1:-1])
    wc = 0.5 * (w[1:-1, 1:-1, 1:-1] + w[:-2, 1:-1, 1:-1])
    import oracle
    dzf = oracle.Case(32, 32, 32).dzf_global[1:-1]
    coarse = np.zeros((1, 16, 16, 16, 16))
    for c, f in enumerate((uc, vc, wc)):
        fw = f * dzf[:, None, None]
        s = fw.reshape(16, 2, 16, 2, 16, 2).sum(axis=(1, 3, 5))
        vol = dzf.reshape(16, 2).sum(axis=1)[:, None, None] * 4
        coarse[0, ..., c] = s / vol
    ref = go.stats(coarse)[0]
    assert rel(st, ref) < 1e-5


def test_propose_into_channel():
    g, _ = make_gen()
    for precision in (0, 1):
        ch = _channel(32, 32, 32, precision)
        g.propose(ch, 300.0, seed=3)
        u = ch.download("u")
        assert np.all(np.isfinite(u)) and np.abs(interior(u)).max() > 0
        assert ch.check()[2][0] < (1e-12 if precision == 0 else 1e-3)
        w = ch.download("w")
        assert np.all(w[-2] == 0)  # top wall face
        ch.step(5)  # and the solver runs from it
        assert ch.check()[0]
