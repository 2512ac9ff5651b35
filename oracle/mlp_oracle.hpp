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

// sin(pi x) and cos(pi x) rounded to FP32: x is first reduced exactly modulo 2 (an FP32 x is
// exact in double, and so is the remainder), multiples of 1/2 give exact 0 / +-1, any other x
// the double-precision sine and cosine of pi times the remainder.
inline void sincospi_f32(float x, double* s, double* c) {
  double r = std::fmod(double(x), 2.0);
  if (r < 0.0) r += 2.0;
  if (r * 2.0 == std::floor(r * 2.0)) {  // r in {0, 0.5, 1, 1.5}
    static const double ks[4] = {0.0, 1.0, 0.0, -1.0}, kc[4] = {1.0, 0.0, -1.0, 0.0};
    const int q = int(r * 2.0);
    *s = ks[q];
    *c = kc[q];
    return;
  }
  *s = double(float(std::sin(M_PI * r)));
  *c = double(float(std::cos(M_PI * r)));
}

// Features of one record: sin/cos(pi * x * 2^j) of the normalised position, j < 12, then
// wo, n, albedo, roughness.
inline void encode(const float* rec, const float* lo, const float* inv_ext, double* f) {
  for (int a = 0; a < 3; ++a) {
    float x = (rec[a] - lo[a]) * inv_ext[a];
    for (int j = 0; j < 12; ++j) {
      sincospi_f32(x, &f[a * 24 + 2 * j], &f[a * 24 + 2 * j + 1]);
      x = x * 2.0f;
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
