// mlp_oracle.hpp — TEST INFRASTRUCTURE, NOT THE PRODUCT.
//
// CPU restatement of the radiance cache's network (the reference has no learned component;
// this is the checker the GPU's forward pass, gradients and Adam steps are compared with).
// Two modes:
//   emulate = true : the GPU's arithmetic — BF16 inputs, weights, activations and layer
//                    gradients (round to nearest even), FP32 results of each dot product;
//   emulate = false: plain FP64, for finite-difference checks of the gradient formulas.
// Network: 82 features (+14 zero pads) -> 5 x 64 ReLU -> 3 (+13 zero pads), no biases;
// weights row-major out x in per layer at offsets 0, 6144, 10240, 14336, 18432, 22528.
// Loss: mean over samples and channels of (o - t)^2 / (o^2 + 0.01), denominator constant.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace oracle {
namespace mlp {

constexpr int kIn = 82, kInPad = 96, kHidden = 64, kLayers = 6, kOut = 3, kOutPad = 16, kRecord = 16;
constexpr int kParams = 23552;
inline int layer_k(int l) { return l == 0 ? kInPad : kHidden; }
inline int layer_n(int l) { return l == kLayers - 1 ? kOutPad : kHidden; }
inline int layer_off(int l) {
  static const int off[6] = {0, 6144, 10240, 14336, 18432, 22528};
  return off[l];
}

inline float bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return f;  // inf / nan unchanged
  u += 0x7FFFu + ((u >> 16) & 1u);
  u &= 0xFFFF0000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

// The network's sin(pi x) / cos(pi x) (the library's own method, restated): x reduced to
// t in [-1/4, 1/4] and a quadrant q (k = rint(x / 2), r = x - 2k, q = rint(2r), t = r - q/2),
// Taylor polynomials of sin(pi t) to t^9 and cos(pi t) to t^10 in Horner form with FP32
// coefficients (-1)^k pi^(2k+1) / (2k+1)! and (-1)^k pi^(2k) / (2k)!, every product and sum
// rounded to FP32 (no contraction: this file is built with -ffp-contract=off), then the
// quadrant. The GPU performs the same operations, so the bits agree.
inline void sincospi_poly(float x, float* s, float* c) {
  const float k = std::rint(x * 0.5f);
  const float r = x - k * 2.0f;
  const float q = std::rint(r * 2.0f);
  const float t = r - q * 0.5f;
  const float t2 = t * t;
  // (-1)^k pi^(2k+1) / (2k+1)!, k = 0..4, and (-1)^k pi^(2k) / (2k)!, k = 0..5, rounded to FP32
  const float sc[5] = {0x1.921fb6p+1f, -0x1.4abbcep+2f, 0x1.466bc6p+1f, -0x1.32d2ccp-1f, 0x1.507834p-4f};
  const float cc[6] = {1.0f, -0x1.3bd3ccp+2f, 0x1.03c1f0p+2f, -0x1.55d3c8p+0f, 0x1.e1f506p-3f, -0x1.a6d1f2p-6f};
  float ps = sc[4];
  for (int i = 3; i >= 0; --i) ps = ps * t2 + sc[i];
  const float st = ps * t;
  float pc = cc[5];
  for (int i = 4; i >= 0; --i) pc = pc * t2 + cc[i];
  const float ct = pc;
  switch (int(q) & 3) {
    case 0: *s = st; *c = ct; break;
    case 1: *s = ct; *c = -st; break;
    case 2: *s = -st; *c = -ct; break;
    default: *s = -ct; *c = st; break;
  }
}

// Features of one record: sin/cos(pi * x * 2^j) of the normalised position, j < 12 (the
// first band by sincospi_poly, each next one by the double-angle formulas sin 2a = 2 sin a
// cos a, cos 2a = (cos a - sin a)(cos a + sin a) in FP32), then wo, n, albedo, roughness.
inline void encode(const float* rec, const float* lo, const float* inv_ext, double* f) {
  for (int a = 0; a < 3; ++a) {
    float s, c;
    sincospi_poly((rec[a] - lo[a]) * inv_ext[a], &s, &c);
    for (int j = 0; j < 12; ++j) {
      f[a * 24 + 2 * j] = s;
      f[a * 24 + 2 * j + 1] = c;
      const float s2 = (s * c) * 2.0f;
      c = (c - s) * (c + s);
      s = s2;
    }
  }
  f[72] = rec[4]; f[73] = rec[5]; f[74] = rec[6];
  f[75] = rec[8]; f[76] = rec[9]; f[77] = rec[10];
  f[78] = rec[12]; f[79] = rec[13]; f[80] = rec[14];
  f[81] = rec[3];
  for (int k = kIn; k < kInPad; ++k) f[k] = 0.0;
}

struct Net {
  std::vector<double> w;  // kParams, possibly BF16-rounded
  bool emulate;
  Net(const float* weights, bool emu) : w(kParams), emulate(emu) {
    for (int p = 0; p < kParams; ++p) w[p] = emu ? double(bf16(weights[p])) : double(weights[p]);
  }
  double q(double x) const { return emulate ? double(bf16(float(x))) : x; }
  double fin(double x) const { return emulate ? double(float(x)) : x; }

  // How far an FP32 value v lies from the nearest BF16 rounding boundary (the midpoint
  // between the two BF16 neighbours of v), in units of 2^-24 * s: s is the sum of the
  // magnitudes of the terms that produced v (|v| for a single rounded value), so an FP32
  // result computed in another order, within k * 2^-24 * s of this one, rounds to the same
  // BF16 value whenever the margin exceeds k.
  static double bf16_margin(double v, double s) {
    const float f = float(v);
    if (f == 0.f || !std::isfinite(f) || s <= 0.0) return 1e300;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    const uint32_t lo_bits = u & 0xFFFF0000u, hi_bits = lo_bits + 0x10000u;
    float lo, hi;
    std::memcpy(&lo, &lo_bits, 4);
    std::memcpy(&hi, &hi_bits, 4);
    const double mid = 0.5 * (double(lo) + double(hi));
    return std::fabs(v - mid) / (std::ldexp(1.0, -24) * s);
  }

  // acts[l] = input of layer l (acts[0] = features), out = 16 outputs. In emulate mode,
  // `margin` (optional) receives the smallest bf16_margin of every value the forward pass
  // rounds to BF16 (the features and the five hidden layers' pre-activations that pass the
  // ReLU), and `out_scale` (optional, 16) the sums of the output terms' magnitudes.
  void forward(const double* feat, std::vector<std::vector<double>>& acts, double* out, double* margin = nullptr,
               double* out_scale = nullptr) const {
    acts.assign(kLayers, {});
    acts[0].resize(kInPad);
    double mg = 1e300;
    for (int k = 0; k < kInPad; ++k) {
      acts[0][k] = q(feat[k]);
      if (margin) mg = std::min(mg, bf16_margin(feat[k], std::fabs(feat[k])));
    }
    for (int l = 0; l < kLayers; ++l) {
      const int K = layer_k(l), N = layer_n(l);
      std::vector<double> y(N), mag(N);
      for (int o = 0; o < N; ++o) {
        double s = 0.0, m = 0.0;
        for (int i = 0; i < K; ++i) {
          const double t = w[layer_off(l) + o * K + i] * acts[l][i];
          s += t;
          m += std::fabs(t);
        }
        y[o] = fin(s);
        mag[o] = m;
      }
      if (l + 1 < kLayers) {
        acts[l + 1].resize(N);
        for (int o = 0; o < N; ++o) {
          acts[l + 1][o] = q(y[o] > 0.0 ? y[o] : 0.0);
          if (margin && y[o] > 0.0) mg = std::min(mg, bf16_margin(y[o], mag[o]));
        }
      } else {
        for (int o = 0; o < N; ++o) {
          out[o] = y[o];
          if (out_scale) out_scale[o] = mag[o];
        }
      }
    }
    if (margin) *margin = mg;
  }

  // Adds this sample's gradient (scaled) to grad; returns its loss sum over channels.
  double backward(const double* feat, const float* target, double scale, double* grad) const {
    std::vector<std::vector<double>> acts;
    double out[kOutPad];
    forward(feat, acts, out);
    double loss = 0.0;
    std::vector<double> G(kOutPad, 0.0);
    for (int c = 0; c < kOut; ++c) {
      const double o = emulate ? double(float(out[c])) : out[c];
      const double d = o - double(target[c]);
      const double wgt = emulate ? double(1.0f / (float(o) * float(o) + 0.01f)) : 1.0 / (o * o + 0.01);
      loss += d * d * wgt;
      G[c] = q(emulate ? double(2.0f * float(d) * float(wgt) * float(scale)) : 2.0 * d * wgt * scale);
    }
    for (int l = kLayers - 1; l >= 0; --l) {
      const int K = layer_k(l), N = layer_n(l);
      for (int o = 0; o < N; ++o)
        for (int i = 0; i < K; ++i) grad[layer_off(l) + o * K + i] += G[o] * acts[l][i];
      if (l == 0) break;
      std::vector<double> gp(K);
      for (int i = 0; i < K; ++i) {
        double s = 0.0;
        for (int o = 0; o < N; ++o) s += G[o] * w[layer_off(l) + o * K + i];
        s = fin(s);
        gp[i] = q(acts[l][i] > 0.0 ? s : 0.0);
      }
      G = gp;
    }
    return loss;
  }
};

inline void adam(float* w, float* m, float* v, const float* g, uint32_t step, float lr, float b1, float b2, float eps) {
  const float c1 = 1.0f - std::pow(b1, float(step)), c2 = 1.0f - std::pow(b2, float(step));
  for (int p = 0; p < kParams; ++p) {
    m[p] = b1 * m[p] + (1.0f - b1) * g[p];
    v[p] = b2 * v[p] + (1.0f - b2) * g[p] * g[p];
    w[p] = w[p] - lr * (m[p] / c1) / (std::sqrt(v[p] / c2) + eps);
  }
}

}  // namespace mlp
}  // namespace oracle
