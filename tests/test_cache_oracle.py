"""CPU checks of the radiance cache's oracle network and its host-side constants."""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT
from pbrt_b200 import _capi
from pbrt_b200.cache import PARAMS, RECORD, random_records

BOUNDS = np.array([-1, -1, -1, 1, 1, 1], np.float32)


def _problem(n=40, seed=0):
    r = random_records(n, BOUNDS[:3], BOUNDS[3:], seed=seed)
    w = ((np.random.default_rng(seed).random(PARAMS) - 0.5) * 0.2).astype(np.float32)
    t = np.random.default_rng(seed + 1).random((n, 3)).astype(np.float32)
    return w, r, t


def test_header_constants_match():
    h = open(f"{ROOT}/include/pbrt_b200.h").read()
    assert int(re.search(r"#define PBRT_CACHE_PARAMS (\d+)u", h).group(1)) == PARAMS == oracle.MLP_PARAMS
    assert int(re.search(r"#define PBRT_CACHE_RECORD (\d+)u", h).group(1)) == RECORD
    # u64 + 4 floats + 6 floats + 3 u32, padded to 8
    assert C.sizeof(_capi.CacheParams) == 64


def test_gradient_matches_finite_differences():
    """Exact (FP64) mode: the analytic gradient equals central differences of the loss with
    the relative-L2 denominator held at its unperturbed value, the loss the gradient is of."""
    w, r, t = _problem()
    g, loss = oracle.mlp_gradient(w, BOUNDS, r, t, emulate=False)
    o0 = oracle.mlp_forward_f64(w, BOUNDS, r)
    den = o0 * o0 + 0.01
    assert loss == pytest.approx(np.mean((o0 - t) ** 2 / den), rel=1e-12)

    def frozen(ww):
        o = oracle.mlp_forward_f64(ww, BOUNDS, r)
        return np.mean((o - t) ** 2 / den)

    rng = np.random.default_rng(7)
    offs = [0, 6144, 10240, 14336, 18432, 22528, 23552]
    for layer in range(6):
        rows = 3 if layer == 5 else (offs[layer + 1] - offs[layer]) // (96 if layer == 0 else 64)
        k = 82 if layer == 0 else 64
        kk = 96 if layer == 0 else 64
        for _ in range(3):
            p = offs[layer] + int(rng.integers(rows)) * kk + int(rng.integers(k))
            fds = []
            for h in (1e-5, 2e-6):  # two steps: a ReLU kink inside one interval spoils only it
                wp, wm = w.copy(), w.copy()
                wp[p] += np.float32(h)
                wm[p] -= np.float32(h)
                fds.append((frozen(wp) - frozen(wm)) / (float(wp[p]) - float(wm[p])))
            assert any(fd == pytest.approx(g[p], rel=1e-5, abs=1e-10) for fd in fds), (layer, p, g[p], fds)


def test_padding_rows_and_columns_get_no_gradient():
    w, r, t = _problem()
    g, _ = oracle.mlp_gradient(w, BOUNDS, r, t, emulate=True)
    first = g[:6144].reshape(64, 96)
    assert np.all(first[:, 82:] == 0.0)  # zero-padded features
    last = g[22528:].reshape(16, 64)
    assert np.all(last[3:] == 0.0)  # padded outputs carry no loss


def test_emulated_forward_close_to_exact():
    w, r, _ = _problem(200)
    e = oracle.mlp_forward(w, BOUNDS, r, emulate=True)
    x = oracle.mlp_forward_f64(w, BOUNDS, r)
    scale = np.abs(x).max()
    assert np.abs(e - x).max() < 0.05 * scale


def test_adam_formula():
    rng = np.random.default_rng(3)
    w = rng.standard_normal(PARAMS).astype(np.float32)
    m = (rng.standard_normal(PARAMS) * 0.01).astype(np.float32)
    v = (rng.random(PARAMS) * 0.01).astype(np.float32)
    g = rng.standard_normal(PARAMS).astype(np.float32)
    w0, m0, v0 = w.copy(), m.copy(), v.copy()
    oracle.mlp_adam(w, m, v, g, 3, 1e-2, 0.9, 0.99, 1e-8)
    f = np.float32
    c1, c2 = f(1) - f(0.9) ** f(3), f(1) - f(0.99) ** f(3)
    mm = f(0.9) * m0 + (f(1) - f(0.9)) * g
    vv = f(0.99) * v0 + (f(1) - f(0.99)) * g * g
    np.testing.assert_array_equal(m, mm)
    np.testing.assert_array_equal(v, vv)
    np.testing.assert_allclose(w, w0 - f(1e-2) * (mm / c1) / (np.sqrt(vv / c2) + f(1e-8)), rtol=1e-6)


def _emulated_bands(x):
    """The position encoding's documented FP32 operations, emulated in numpy float32: one
    polynomial sin / cos (pi x) (reduction to |t| <= 1/4 and a quadrant, Taylor coefficients
    rounded to FP32, Horner with rounded multiplies and adds), then double-angle octaves."""
    f = np.float32
    sc = [f(float.fromhex(h)) for h in ("0x1.921fb6p+1", "-0x1.4abbcep+2", "0x1.466bc6p+1", "-0x1.32d2ccp-1",
                                        "0x1.507834p-4")]
    cc = [f(float.fromhex(h)) for h in ("0x1p+0", "-0x1.3bd3ccp+2", "0x1.03c1f0p+2", "-0x1.55d3c8p+0",
                                        "0x1.e1f506p-3", "-0x1.a6d1f2p-6")]
    x = x.astype(np.float32)
    k = np.rint(x * f(0.5)).astype(np.float32)
    r = (x - k * f(2)).astype(np.float32)
    q = np.rint(r * f(2)).astype(np.float32)
    t = (r - q * f(0.5)).astype(np.float32)
    t2 = (t * t).astype(np.float32)
    ps = np.full_like(t, sc[4])
    for c in sc[3::-1]:
        ps = ((ps * t2).astype(np.float32) + c).astype(np.float32)
    st = (ps * t).astype(np.float32)
    pc = np.full_like(t, cc[5])
    for c in cc[4::-1]:
        pc = ((pc * t2).astype(np.float32) + c).astype(np.float32)
    qi = q.astype(np.int64) & 3
    s = np.select([qi == 0, qi == 1, qi == 2], [st, pc, -st], -pc).astype(np.float32)
    c = np.select([qi == 0, qi == 1, qi == 2], [pc, -st, -pc], st).astype(np.float32)
    bands = []
    for _ in range(12):
        bands += [s, c]
        s, c = ((s * c).astype(np.float32) * f(2)).astype(np.float32), ((c - s) * (c + s)).astype(np.float32)
    return np.stack(bands, axis=1)


def test_position_encoding_pinned():
    """The oracle's position features equal, bit for bit, an independent numpy emulation of
    the documented FP32 operations, and stay within 1.5e-7 of sin / cos (pi 2^j x) at the
    first band and 2^j x 3e-7 at band j (each double-angle step doubles the error it carries
    and adds about one rounding)."""
    r = random_records(20000, BOUNDS[:3], BOUNDS[3:], seed=5)
    r[:64, 0] = np.linspace(-1.0, 1.0, 64, dtype=np.float32)  # quadrant edges: x = 0, 1/4, 1/2, ...
    feat = oracle.mlp_encode(BOUNDS, r)
    x = ((r[:, :3] - BOUNDS[:3]) * (np.float32(1) / (BOUNDS[3:] - BOUNDS[:3]))).astype(np.float32)
    for a in range(3):
        got = feat[:, 24 * a:24 * a + 24]
        assert np.array_equal(got.view(np.uint32), _emulated_bands(x[:, a]).view(np.uint32))
        for j in range(12):
            ang = np.pi * x[:, a].astype(np.float64) * 2.0 ** j
            err = max(np.abs(got[:, 2 * j] - np.sin(ang)).max(), np.abs(got[:, 2 * j + 1] - np.cos(ang)).max())
            assert err <= (1.5e-7 if j == 0 else 2.0 ** j * 3e-7), (a, j, err)
    assert np.array_equal(feat[:, 72:75], r[:, 4:7]) and np.array_equal(feat[:, 81], r[:, 3])
