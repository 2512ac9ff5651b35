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
