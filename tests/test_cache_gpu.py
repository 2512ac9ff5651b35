"""Radiance-cache network on the GPU against the oracle network (BF16-emulating mode).

Forward and gradient are not bit-exact: the tensor cores sum in another order than the
oracle, so an FP32 pre-activation near a BF16 rounding boundary can round the other way.
The tolerances below bound that; the Adam step, which has no such freedom, is bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from pbrt_b200 import PbrtError
from pbrt_b200.cache import PARAMS, RadianceCache, random_records

pytestmark = pytest.mark.gpu

LO, HI = (-1.0, -0.5, -2.0), (1.0, 1.5, 0.0)
BOUNDS = np.array(LO + HI, np.float32)
OFFS = [0, 6144, 10240, 14336, 18432, 22528, 23552]


@pytest.fixture(scope="module")
def cache():
    c = RadianceCache(LO, HI, seed=5)
    yield c
    c.close()


def _targets(records):
    # a smooth radiance-like function of position, normal and albedo
    p, n, a = records[:, 0:3], records[:, 8:11], records[:, 12:15]
    shade = 0.6 + 0.4 * n[:, 1:2] + 0.2 * np.sin(3.0 * p[:, 0:1])
    return (a * shade).astype(np.float32)


def test_initial_weights_are_seeded(cache):
    w = cache.weights()
    assert w.shape == (PARAMS,) and np.all(np.isfinite(w))
    first = w[:6144].reshape(64, 96)
    assert np.all(first[:, 82:] == 0.0)
    assert np.all(w[22528:].reshape(16, 64)[3:] == 0.0)
    other = RadianceCache(LO, HI, seed=5)
    np.testing.assert_array_equal(other.weights(), w)
    third = RadianceCache(LO, HI, seed=6)
    assert not np.array_equal(third.weights(), w)


# A BF16-rounded value whose FP32 margin to a rounding boundary (in units of 2^-24 times the
# magnitude sum of its terms) exceeds MARGIN rounds identically on the GPU and in the oracle,
# whatever their summation orders: two FP32 orders of a 96-term sum differ by far less. A row
# whose every rounded value clears it has bit-identical activations on both sides, so its
# outputs differ only by the last layer's FP32 summation order: at most 2 * 64 * 2^-24 times
# the output's magnitude sum.
MARGIN, OUT_UNITS = 16.0, 128.0


@pytest.mark.parametrize("n", [1, 127, 1000, 40_000])
def test_forward_matches_oracle(cache, n):
    cache.reset()
    r = random_records(n, LO, HI, seed=n)
    got = cache.query(r)
    want, margin, scale = oracle.mlp_forward_margins(cache.weights(), BOUNDS, r)
    clear = margin > MARGIN
    bound = OUT_UNITS * 2.0 ** -24 * scale
    err = np.abs(got.astype(np.float64) - want)
    bad = clear[:, None] & (err > bound)
    assert not bad.any(), f"{int(bad.any(axis=1).sum())} of {int(clear.sum())} clear rows differ beyond FP32 order"
    # rows near a rounding boundary may take the other BF16 value there: at most one BF16 ulp
    # somewhere in the network, so their error stays small
    near = ~clear
    if near.any():
        rel = err[near] / max(float(np.abs(want).max()), 1e-3)
        assert rel.max() < 3e-2 and np.median(rel) < 2e-3


def test_forward_bit_exact_on_an_exact_network():
    """Weights in {0, +-1} (two per row), positions on half units (every sin/cos feature is
    exactly 0 or +-1) and the other features in {0, +-1}: every product and sum is a small
    integer, exact in any order, and every activation is exact in BF16, so the GPU's output
    must equal the oracle's exactly on every row (all six tcgen05 layers, every tile row)."""
    rng = np.random.default_rng(7)
    w = np.zeros(PARAMS, np.float32)
    for layer in range(6):
        k = 96 if layer == 0 else 64
        rows = 16 if layer == 5 else 64
        used = 82 if layer == 0 else 64
        blk = w[OFFS[layer]:OFFS[layer + 1]].reshape(rows, k)
        for o in range(3 if layer == 5 else rows):
            cols = rng.choice(used, size=2, replace=False)
            blk[o, cols] = rng.choice([-1.0, 1.0], size=2)
    c = RadianceCache((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), seed=1)
    try:
        c.set_weights(w)
        n = 3000
        r = np.zeros((n, 16), np.float32)
        r[:, 0:3] = rng.integers(0, 3, size=(n, 3)) * 0.5
        for cols in ((3,), (4, 5, 6), (8, 9, 10), (12, 13, 14)):
            r[:, list(cols)] = rng.integers(-1, 2, size=(n, len(cols)))
        got = c.query(r)
        want = oracle.mlp_forward(w, np.array([0, 0, 0, 1, 1, 1], np.float32), r, emulate=True)
        assert np.all(np.abs(want) <= 64) and np.any(want != 0)
        np.testing.assert_array_equal(got, want)
    finally:
        c.close()


def test_gradient_matches_oracle(cache):
    cache.reset()
    n = 1000  # ragged last tile
    r = random_records(n, LO, HI, seed=11)
    t = _targets(r)
    g, loss = cache.gradient(r, t)
    go, lo = oracle.mlp_gradient(cache.weights(), BOUNDS, r, t, emulate=True)
    assert loss == pytest.approx(lo, rel=2e-2)
    for layer in range(6):
        a, b = g[OFFS[layer]:OFFS[layer + 1]], go[OFFS[layer]:OFFS[layer + 1]]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert rel < 3e-2, (layer, rel)
    assert np.all(g[:6144].reshape(64, 96)[:, 82:] == 0.0)
    assert np.all(g[22528:].reshape(16, 64)[3:] == 0.0)


def test_gradient_is_deterministic(cache):
    cache.reset()
    r = random_records(5000, LO, HI, seed=12)
    t = _targets(r)
    g1, _ = cache.gradient(r, t)
    g2, _ = cache.gradient(r, t)
    np.testing.assert_array_equal(g1, g2)


def test_adam_step_bit_exact(cache):
    cache.reset()
    r = random_records(3000, LO, HI, seed=13)
    t = _targets(r)
    w0 = cache.weights()
    g, _ = cache.gradient(r, t)
    cache.train_step(r, t)
    w1 = cache.weights()
    w, m, v = w0.copy(), np.zeros(PARAMS, np.float32), np.zeros(PARAMS, np.float32)
    oracle.mlp_adam(w, m, v, g, 1, 1e-2, 0.9, 0.99, 1e-8)
    np.testing.assert_array_equal(w1, w)


def test_training_reduces_loss(cache):
    cache.reset()
    losses = []
    for step in range(150):
        r = random_records(8192, LO, HI, seed=1000 + step)
        losses.append(cache.train_step(r, _targets(r)))
    assert np.all(np.isfinite(losses))
    assert np.mean(losses[-10:]) < 0.25 * np.mean(losses[:3]), (losses[:3], losses[-10:])
    r = random_records(4096, LO, HI, seed=99)
    t = _targets(r)
    got = cache.query(r)
    assert np.mean((got - t) ** 2 / (t * t + 0.01)) < 0.5


def test_checkpoint_round_trip(cache):
    cache.reset()
    for step in range(3):
        r = random_records(2048, LO, HI, seed=step)
        cache.train_step(r, _targets(r))
    blob = cache.save()
    other = RadianceCache(LO, HI, seed=77)
    other.load(blob)
    np.testing.assert_array_equal(other.weights(), cache.weights())
    q = random_records(500, LO, HI, seed=3)
    np.testing.assert_array_equal(other.query(q), cache.query(q))
    # the Adam state travels too: the next step agrees
    r = random_records(2048, LO, HI, seed=9)
    cache.train_step(r, _targets(r))
    other.train_step(r, _targets(r))
    np.testing.assert_array_equal(other.weights(), cache.weights())
    with pytest.raises(PbrtError):
        other.load(b"\0" * len(blob))
    with pytest.raises(PbrtError):
        other.load(blob[:-4])


def test_set_weights_round_trip(cache):
    w = ((np.random.default_rng(4).random(PARAMS) - 0.5) * 0.1).astype(np.float32)
    cache.set_weights(w)
    np.testing.assert_array_equal(cache.weights(), w)
    r = random_records(300, LO, HI, seed=21)
    want = oracle.mlp_forward(w, BOUNDS, r, emulate=True)
    got = cache.query(r)
    assert np.abs(got - want).max() < 3e-2 * max(float(np.abs(want).max()), 1e-3)


def test_device_buffers_and_alignment(cache):
    torch = pytest.importorskip("torch")
    cache.reset()
    r = random_records(700, LO, HI, seed=31)
    rd = torch.from_numpy(r).cuda()
    out = torch.zeros((700, 3), dtype=torch.float32, device="cuda")
    cache.ctx.check(cache.ctx.lib.pbrt_cache_query(cache.h, rd.data_ptr(), 700, out.data_ptr()), "query")
    np.testing.assert_array_equal(out.cpu().numpy(), cache.query(r))
    flat = torch.zeros(700 * 16 + 1, dtype=torch.float32, device="cuda")
    rc = cache.ctx.lib.pbrt_cache_query(cache.h, flat.data_ptr() + 4, 700, out.data_ptr())
    assert rc == 1  # misaligned device records are refused, not read
