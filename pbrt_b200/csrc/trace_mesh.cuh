// trace_mesh.cuh — nearest-hit and any-hit traversal of one triangle mesh's BVH.
//
// Semantics are those of the reference, operation for operation:
//   - slab test: AABoundingBox::hit (src/geom/aabound.rs:323-355), widened by 2γ(3);
//   - nearest hit: BVHTree::traverse (src/shapes/triangle_mesh/bvh.rs:450-526): the root
//     box is tested once, each child box once by its parent, the nearer child is visited
//     first (the right one only when strictly nearer), a popped node is dropped when its
//     entry distance is >= the nearest hit so far, and a triangle replaces the current
//     hit only when t < min_t and near <= t <= far;
//   - any hit: BVHTree::intersect_p (bvh.rs:381-420), first valid hit ends the ray;
//   - triangle test: Möller–Trumbore as intersect_ray (triangle_mesh.rs:183-217).
// Because the tree, the visiting order and every rounding match, the returned triangle
// and t are bit-identical to the FP32 restatement of the reference.
//
// Layout (mesh_bvh.hpp): nodes are 32-byte records read as two float4 (bmin|left_first,
// bmax|count); a sibling pair is one aligned 64-byte read
// (two 256-bit loads); triangles are three SoA
// streams in leaf order.
#pragma once

#include <cfloat>

#include "device_math.cuh"

namespace pbrt {

constexpr int kTraceStack = 64;  // scenes whose trees are deeper are refused at creation

enum DeviceError : uint32_t {
  kErrBudget = 1u,  // a traversal exceeded its iteration budget (malformed tree)
  kErrStack = 2u,   // a traversal stack would have overflowed
  kErrCopy = 8u,    // a wait for a bulk copy into shared memory ran out of its budget
};

// One 32-byte node record (bmin|left_first, bmax|count) as a single 256-bit load. Node
// arrays come from cudaMalloc and records are 32 bytes, so every record is 32-byte aligned.
PBRT_DEV void load_node(const float4* p, float4& lo, float4& hi) {
  asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=f"(lo.x), "=f"(lo.y), "=f"(lo.z), "=f"(lo.w), "=f"(hi.x), "=f"(hi.y), "=f"(hi.z), "=f"(hi.w)
      : "l"(p));
}

struct MeshView {
  const float4* nodes;  // 2 float4 per node
  const float4* tri_a;
  const float4* tri_b;
  const float2* tri_c;
  uint32_t node_count;  // GPU numbering, including the padding slot
};

// A ray prepared for box tests: the reciprocals depend on the ray alone (the reference
// hoists them by inlining, aabound.rs:316-321), and which slab plane is entered first is
// fixed by the sign of each reciprocal (the swap at aabound.rs:338-340).
struct PRay {
  F3 o, d, inv;
  uint32_t neg;   // bit a: inv[a] < 0
  uint32_t zero;  // bit a: d[a] == 0 (slab parallel to the ray)
};

PBRT_DEV PRay prepare_ray(const F3& o, const F3& d) {
  PRay r;
  r.o = o;
  r.d = d;
  r.inv = mk3(frcp(d.x), frcp(d.y), frcp(d.z));
  r.neg = (r.inv.x < 0.f ? 1u : 0u) | (r.inv.y < 0.f ? 2u : 0u) | (r.inv.z < 0.f ? 4u : 0u);
  r.zero = (d.x == 0.f ? 1u : 0u) | (d.y == 0.f ? 2u : 0u) | (d.z == 0.f ? 4u : 0u);
  return r;
}

// One slab of AABoundingBox::hit. Once tmax < tmin it stays so (tmin only grows, tmax
// only shrinks, fmaxf/fminf never return NaN here), so testing once at the end gives the
// reference's early-exit answer.
PBRT_DEV void slab_axis(float o, float inv, bool neg, bool zero, float lo, float hi, float& tmin, float& tmax,
                        bool& miss) {
  if (zero) {
    if (o < lo || o > hi) miss = true;
    return;
  }
  const float W = PBRT_SLAB_WIDENING_F32;
  float t0 = fm(fs(neg ? hi : lo, o), inv);
  float t1 = fm(fs(neg ? lo : hi, o), inv);
  t0 = fs(t0, fm(fabsf(t0), W));
  t1 = fa(t1, fm(fabsf(t1), W));
  tmin = fmaxf(t0, tmin);
  tmax = fminf(t1, tmax);
}

// One slab with no parallel axis: the branch-free form used whenever no direction
// component is zero (every incoherent ray in practice).
PBRT_DEV void slab_axis_fast(float o, float inv, bool neg, float lo, float hi, float& tmin, float& tmax) {
  const float W = PBRT_SLAB_WIDENING_F32;
  float t0 = fm(fs(neg ? hi : lo, o), inv);
  float t1 = fm(fs(neg ? lo : hi, o), inv);
  t0 = fs(t0, fm(fabsf(t0), W));
  t1 = fa(t1, fm(fabsf(t1), W));
  tmin = fmaxf(t0, tmin);
  tmax = fminf(t1, tmax);
}

PBRT_DEV bool box_hit(const PRay& r, const float4& lo, const float4& hi, float tmin, float tmax, float& entry) {
  if (r.zero == 0u) {
    slab_axis_fast(r.o.x, r.inv.x, r.neg & 1u, lo.x, hi.x, tmin, tmax);
    slab_axis_fast(r.o.y, r.inv.y, r.neg & 2u, lo.y, hi.y, tmin, tmax);
    slab_axis_fast(r.o.z, r.inv.z, r.neg & 4u, lo.z, hi.z, tmin, tmax);
    entry = tmin;
    return !(tmax < tmin);
  }
  bool miss = false;
  slab_axis(r.o.x, r.inv.x, r.neg & 1u, r.zero & 1u, lo.x, hi.x, tmin, tmax, miss);
  slab_axis(r.o.y, r.inv.y, r.neg & 2u, r.zero & 2u, lo.y, hi.y, tmin, tmax, miss);
  slab_axis(r.o.z, r.inv.z, r.neg & 4u, r.zero & 4u, lo.z, hi.z, tmin, tmax, miss);
  entry = tmin;
  return !miss && !(tmax < tmin);
}

// Möller–Trumbore with e1, e2 precomputed (bit-identical to forming them here).
PBRT_DEV bool tri_hit(const PRay& r, const float4& A, const float4& B, float e2z, float& t) {
  const F3 p0 = mk3(A.x, A.y, A.z);
  const F3 e1 = mk3(A.w, B.x, B.y);
  const F3 e2 = mk3(B.z, B.w, e2z);
  const F3 pv = cross3(r.d, e2);
  const float det = dot3(e1, pv);
  if (fabsf(det) < 1e-8f) return false;
  const float inv_det = frcp(det);
  const F3 s = sub3(r.o, p0);
  const float u = fm(inv_det, dot3(s, pv));
  if (u < 0.f || u > 1.f) return false;
  const F3 q = cross3(s, e1);
  const float v = fm(inv_det, dot3(r.d, q));
  if (v < 0.f || fa(u, v) > 1.f) return false;
  t = fm(inv_det, dot3(e2, q));
  return true;
}

struct TraceCounters {
  uint32_t nodes_visited, box_tests, triangle_tests;
};

// Nearest hit of one ray against one mesh. Returns the original triangle index or
// 0xFFFFFFFF; *t_out holds the hit distance (FLT_MAX-initialised min_t otherwise).
template <bool kCount>
PBRT_DEV uint32_t mesh_closest(const MeshView& m, const PRay& r, float near, float far, float* t_out,
                               TraceCounters* cnt, uint32_t* err) {
  float min_t = FLT_MAX;
  uint32_t best = 0xFFFFFFFFu;
  const float4 rlo = __ldg(&m.nodes[0]);
  const float4 rhi = __ldg(&m.nodes[1]);
  float entry;
  if (kCount) cnt->box_tests++;
  // The root is pushed, then dropped at pop if its entry is >= min_t = FLT_MAX (bvh.rs:462-472).
  if (box_hit(r, rlo, rhi, near, far, entry) && entry < FLT_MAX) {
    uint32_t lf = __float_as_uint(rlo.w), count = __float_as_uint(rhi.w);
    uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
    float stk_e[kTraceStack];
    int sp = 0;
    uint32_t budget = m.node_count;
    for (;;) {
      if (budget-- == 0) {
        atomicOr(err, kErrBudget);
        break;
      }
      if (kCount) cnt->nodes_visited++;
      bool pop = true;
      if (count > 0) {
        for (uint32_t k = lf; k < lf + count; ++k) {
          const float4 A = __ldg(&m.tri_a[k]);
          const float4 B = __ldg(&m.tri_b[k]);
          const float2 C = __ldg(&m.tri_c[k]);
          if (kCount) cnt->triangle_tests++;
          float t;
          if (tri_hit(r, A, B, C.x, t) && t < min_t && t >= near && t <= far) {
            min_t = t;
            best = __float_as_uint(C.y);
          }
        }
      } else {
        float4 l0, l1, r0, r1;
        load_node(&m.nodes[2 * lf], l0, l1);
        load_node(&m.nodes[2 * lf + 2], r0, r1);
        float dl, dr;
        if (kCount) cnt->box_tests += 2;
        const bool hl = box_hit(r, l0, l1, near, far, dl);
        const bool hr = box_hit(r, r0, r1, near, far, dr);
        const bool swap = hl && hr && dr < dl;  // right first only when strictly nearer
        const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
        const float dn = swap ? dr : dl, df = swap ? dl : dr;
        const float4 n0 = swap ? r0 : l0, n1 = swap ? r1 : l1;
        const float4 f0 = swap ? l0 : r0, f1 = swap ? l1 : r1;
        const bool take_f = hf && df < min_t;
        const bool take_n = hn && dn < min_t;
        if (take_n) {
          if (take_f) {
            if (sp >= kTraceStack) {
              atomicOr(err, kErrStack);
              break;
            }
            stk_lf[sp] = __float_as_uint(f0.w);
            stk_cnt[sp] = __float_as_uint(f1.w);
            stk_e[sp] = df;
            ++sp;
          }
          lf = __float_as_uint(n0.w);
          count = __float_as_uint(n1.w);
          pop = false;
        } else if (take_f) {
          lf = __float_as_uint(f0.w);
          count = __float_as_uint(f1.w);
          pop = false;
        }
      }
      if (pop) {
        bool found = false;
        while (sp > 0) {
          --sp;
          if (stk_e[sp] < min_t) {
            lf = stk_lf[sp];
            count = stk_cnt[sp];
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  *t_out = min_t;
  return best;
}

// Any hit of one ray against one mesh within [near, far].
PBRT_DEV bool mesh_any(const MeshView& m, const PRay& r, float near, float far, uint32_t* err) {
  const float4 rlo = __ldg(&m.nodes[0]);
  const float4 rhi = __ldg(&m.nodes[1]);
  float entry;
  if (!box_hit(r, rlo, rhi, near, far, entry)) return false;
  uint32_t lf = __float_as_uint(rlo.w), count = __float_as_uint(rhi.w);
  uint32_t stk_lf[kTraceStack], stk_cnt[kTraceStack];
  int sp = 0;
  uint32_t budget = m.node_count;
  for (;;) {
    if (budget-- == 0) {
      atomicOr(err, kErrBudget);
      return false;
    }
    bool pop = true;
    if (count > 0) {
      for (uint32_t k = lf; k < lf + count; ++k) {
        const float4 A = __ldg(&m.tri_a[k]);
        const float4 B = __ldg(&m.tri_b[k]);
        const float2 C = __ldg(&m.tri_c[k]);
        float t;
        if (tri_hit(r, A, B, C.x, t) && t >= near && t <= far) return true;
      }
    } else {
      float4 l0, l1, r0, r1;
      load_node(&m.nodes[2 * lf], l0, l1);
      load_node(&m.nodes[2 * lf + 2], r0, r1);
      float dl, dr;
      const bool hl = box_hit(r, l0, l1, near, far, dl);
      const bool hr = box_hit(r, r0, r1, near, far, dr);
      // The answer does not depend on the visiting order; the nearer child goes first
      // because it is the likelier blocker.
      const bool swap = hl && hr && dr < dl;
      const float4 n0 = swap ? r0 : l0, n1 = swap ? r1 : l1;
      const float4 f0 = swap ? l0 : r0, f1 = swap ? l1 : r1;
      const bool hn = swap ? hr : hl, hf = swap ? hl : hr;
      if (hn) {
        if (hf) {
          if (sp >= kTraceStack) {
            atomicOr(err, kErrStack);
            return false;
          }
          stk_lf[sp] = __float_as_uint(f0.w);
          stk_cnt[sp] = __float_as_uint(f1.w);
          ++sp;
        }
        lf = __float_as_uint(n0.w);
        count = __float_as_uint(n1.w);
        pop = false;
      } else if (hf) {
        lf = __float_as_uint(f0.w);
        count = __float_as_uint(f1.w);
        pop = false;
      }
    }
    if (pop) {
      if (sp == 0) return false;
      --sp;
      lf = stk_lf[sp];
      count = stk_cnt[sp];
    }
  }
}

}  // namespace pbrt
