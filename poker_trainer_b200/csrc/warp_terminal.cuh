// Fixed-point terminal evaluation shared by the terminal kernels
// (terminal_fast.cu) and the batched river kernel (batch.cu).
//
// A terminal's opponent reach row is converted to 64-bit fixed point
// (scaled by a power of two chosen from the row's maximum so the row sums
// below 2^62); integer sums are exact and associative, so every sum the
// reference's evaluators need (crates/solver/src/eval.rs:40-379) is a
// difference of two prefixes of one scan over the board's layout:
//   weaker (win)    = G[w] - (card a's weaker part) - (card b's)
//   stronger (lose) = (T - G[s]) - (card a's stronger part) - (card b's)
//   equal (tie)     = (G[s] - G[w]) - ... + identical hand (eval.rs:347-379)
//   fold            = T - (card a total) - (card b total) + identical hand
// Each integer result is converted to f64 once, scaled back, multiplied by
// the payoff and, for float rows, rounded to f32 in the evaluator's own
// combination order (scalar: eval_showdown's two f32 parts; batched:
// showdown_batch's f64 sum).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"

namespace dcfr {

#ifndef WARP_TERMINAL_HANDS_PER_STEP
#define WARP_TERMINAL_HANDS_PER_STEP 4
#endif

__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Fixed-point value of one reach entry: trunc(x * 2^S). Products are exact
// (power-of-two scale, below 2^52).
__device__ __forceinline__ long long fixed(float x, double scale) { return __double2ll_rz((double)x * scale); }
__device__ __forceinline__ long long fixed(double x, double scale) { return __double2ll_rz(x * scale); }

// Scale exponent S of a row whose largest entry is mx: mx * 2^S < 2^51, so a
// row of up to 2048 entries sums below 2^62. For double rows S is capped so
// 2^S stays finite; entries below 2^-1020 of that cap truncate to zero.
__device__ __forceinline__ int scale_exponent(float mx) { return 177 - (int)((__float_as_uint(mx) >> 23) & 0xFF); }
__device__ __forceinline__ int scale_exponent(double mx) {
  const int e = (int)((__double_as_longlong(mx) >> 52) & 0x7FF);
  const int S = 1073 - e;
  return S > 1020 ? 1020 : S;
}
__device__ __forceinline__ float row_max(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double row_max(double a, double b) { return fmax(a, b); }

// The staged layout a warp evaluates against: opponent hand per element,
// per-hand records and segment starts of one (layout, traverser), and the
// traverser's identical-hand map (0xFFFF: none). L = seg[53] elements.
struct WarpLayout {
  const uint16_t* same;
  const uint16_t* cat;
  const uint4* rec;
  const uint16_t* seg;
  int L;
};

// Per-warp prefix storage needed by warp_terminal_task for layouts of up to
// cstride elements: the prefixes (cstride + 1), then, 16-byte aligned, each
// card's segment start prefix and total (52 x 2).
__host__ __device__ constexpr size_t warp_prefix_entries(int cstride) {
  return (((size_t)cstride + 1 + 1) & ~(size_t)1) + 2 * 52;
}

// Asynchronous copy (cp.async, 16-byte chunks through L2) of the reach row
// of `slot` into the warp's shared row; it lands at a later cp.async wait.
template <typename R>
__device__ __forceinline__ void warp_row_prefetch(const FastArgsT<R>& A, uint32_t slot, R* row, int lane) {
  constexpr int PER16 = 16 / (int)sizeof(R);
  const int hpo = (A.p ^ 1) ? A.hp[1] : A.hp[0];
  const char* src = reinterpret_cast<const char*>(A.reach + (size_t)slot * A.stride);
  const uint32_t dst = (uint32_t)__cvta_generic_to_shared(row);
  for (int i = lane; i < hpo / PER16; i += 32)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * (uint32_t)i), "l"(src + 16 * (size_t)i)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// One terminal task evaluated by one warp (all 32 lanes call it). row is
// the warp's shared copy of the reach row (stride entries), G its prefix
// storage (warp_prefix_entries(cstride) entries, 16-byte aligned). The
// caller has checked the task's slot is live. With PRELOADED the row is
// already in shared memory (warp_row_prefetch, waited for and synced);
// otherwise it is loaded here.
template <typename R, bool PRELOADED = false>
__device__ __forceinline__ void warp_terminal_task(const FastArgsT<R>& A, const FastTask& T, const WarpLayout& Y, R* row,
                                                   long long* G, int lane) {
  constexpr bool F64 = sizeof(R) == 8;
  constexpr int PER16 = 16 / (int)sizeof(R);
  const int p = A.p, o = p ^ 1;
  const int hpo = o ? A.hp[1] : A.hp[0], hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  const int L = Y.L;
  const int E = (((L + 31) >> 5) | 1);  // odd: conflict-free 8-byte strides
  const uint32_t kind = T.kind;
  const bool fold = kind == T_FOLD_SCALAR || kind == T_FOLD_BATCH;
  const bool scalar = kind == T_FOLD_SCALAR || kind == T_SHOWDOWN_SCALAR;
  // 1. Row and its maximum.
  const R* src = A.reach + (size_t)T.slot * A.stride;
  R mx = 0;
  if constexpr (F64) {
    for (int i = lane; i < hpo / PER16; i += 32) {
      double2 v;
      if constexpr (PRELOADED) {
        v = reinterpret_cast<const double2*>(row)[i];
      } else {
        v = reinterpret_cast<const double2*>(src)[i];
        reinterpret_cast<double2*>(row)[i] = v;
      }
      mx = row_max(mx, row_max(v.x, v.y));
    }
  } else {
    for (int i = lane; i < hpo / PER16; i += 32) {
      float4 v;
      if constexpr (PRELOADED) {
        v = reinterpret_cast<const float4*>(row)[i];
      } else {
        v = reinterpret_cast<const float4*>(src)[i];
        reinterpret_cast<float4*>(row)[i] = v;
      }
      mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) mx = row_max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
  const int S = scale_exponent(mx);
  const double scale = pow2(S), inv = pow2(-S);
  const double pa = T.a * inv, pb = T.b * inv, pc = T.c * inv, pd = T.d * inv;
  __syncwarp();
  if (fold) {
    // A fold needs only the total T0 and each card's total (eval_fold,
    // eval.rs:40-64): the same exact integer sums as the scan's, without it.
    long long t0 = 0;
    for (int k = lane; k < Y.seg[1]; k += 32) t0 += fixed(row[Y.cat[k]], scale);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) t0 += __shfl_xor_sync(0xffffffffu, t0, d);
    for (int c = lane; c < 52; c += 32) {
      long long tc = 0;
      for (int k = Y.seg[1 + c]; k < Y.seg[2 + c]; k++) tc += fixed(row[Y.cat[k]], scale);
      G[c] = tc;
    }
    __syncwarp();
    R* out = A.vals + (size_t)T.row * A.stride;
    for (int h = lane; h < hpp; h += 32) {
      R v = 0;
      if (h < np) {
        const uint32_t w = Y.rec[h].w;
        const int a = (int)(w & 0xFF), b = (int)((w >> 8) & 0xFF);
        const uint16_t sm = Y.same[h];
        const long long si = sm == 0xFFFF ? 0ll : fixed(row[sm], scale);
        const long long F = t0 - G[a] - G[b] + si;
        if constexpr (F64) {
          v = pa * (double)F;
        } else {
          v = (scalar && t0 == 0) ? 0.0f : (float)(pa * (double)F);
        }
      }
      out[h] = v;
    }
    __syncwarp();
    return;
  }
  // 2. Elements in layout order, lane sums, exclusive prefixes (four
  // independent elements per step; integer sums are order-free).
  const int k0 = lane * E, k1 = min(L, k0 + E);
  long long local = 0;
  int k = k0;
  for (; k + 4 <= k1; k += 4) {
    const int c0 = Y.cat[k], c1 = Y.cat[k + 1], c2 = Y.cat[k + 2], c3 = Y.cat[k + 3];
    const long long v0 = fixed(row[c0], scale), v1 = fixed(row[c1], scale);
    const long long v2 = fixed(row[c2], scale), v3 = fixed(row[c3], scale);
    G[k] = v0;
    G[k + 1] = v1;
    G[k + 2] = v2;
    G[k + 3] = v3;
    local += (v0 + v1) + (v2 + v3);
  }
  for (; k < k1; k++) {
    const long long v = fixed(row[Y.cat[k]], scale);
    G[k] = v;
    local += v;
  }
  long long inc = local;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  long long acc = inc - local;
  k = k0;
  for (; k + 4 <= k1; k += 4) {
    const long long v0 = G[k], v1 = G[k + 1], v2 = G[k + 2], v3 = G[k + 3];
    G[k] = acc;
    G[k + 1] = acc + v0;
    G[k + 2] = acc + v0 + v1;
    G[k + 3] = acc + v0 + v1 + v2;
    acc += (v0 + v1) + (v2 + v3);
  }
  for (; k < k1; k++) {
    const long long v = G[k];
    G[k] = acc;
    acc += v;
  }
  const long long total = __shfl_sync(0xffffffffu, inc, 31);
  if (lane == 0) G[L] = total;
  __syncwarp();
  // Each card's segment start prefix and total, once per task.
  longlong2* cs = reinterpret_cast<longlong2*>(G + ((L + 2) & ~1));
  for (int c = lane; c < 52; c += 32) {
    const long long s0 = G[Y.seg[1 + c]];
    cs[c] = make_longlong2(s0, G[Y.seg[2 + c]] - s0);
  }
  __syncwarp();
  // 3. Values in hand order.
  const long long T0 = G[Y.seg[1]];
  R* out = A.vals + (size_t)T.row * A.stride;
  R* fout = T.frow != NONE32 ? A.vals + (size_t)T.frow * A.stride : nullptr;
  auto value = [&](int h, R& v, R& fv) {
    v = 0;
    fv = 0;
    if (h < np) {
      const uint4 q = Y.rec[h];
      const int a = (int)(q.w & 0xFF), b = (int)((q.w >> 8) & 0xFF);
      const longlong2 ca = cs[a], cb = cs[b];
      const uint16_t sm = Y.same[h];
      const long long si = sm == 0xFFFF ? 0ll : fixed(row[sm], scale);
      const long long F = T0 - ca.y - cb.y + si;
      if (q.w >> 16) {
        const long long Gw = G[q.x & 0xFFFF], Gs = G[q.x >> 16];
        const long long Gaw = G[q.y & 0xFFFF], Gas = G[q.y >> 16];
        const long long Gbw = G[q.z & 0xFFFF], Gbs = G[q.z >> 16];
        const long long Wn = (Gw + ca.x + cb.x) - Gaw - Gbw;
        const long long Lx = (T0 + Gas + Gbs) - Gs - (ca.x + ca.y) - (cb.x + cb.y);
        const long long eq = (Gs - Gw) - (Gas - Gaw) - (Gbs - Gbw) + si;
        if constexpr (F64) {
          // Double rows: every value in double, no f32 rounding.
          double res = pa * (double)Wn + pb * (double)Lx;
          if (T.c != 0.0) res += pc * (double)eq;
          v = res;
        } else {
          if (scalar) {
            v = (float)(pa * (double)Wn) + (float)(pb * (double)Lx);
          } else {
            double res = pa * (double)Wn;
            res += pb * (double)Lx;
            v = (float)res;
          }
          if (T.c != 0.0) v += (float)(pc * (double)eq);
        }
      }
      if (fout) {
        if constexpr (F64) fv = pd * (double)F;
        else fv = (float)(pd * (double)F);
      }
    }
  };
  // HU hands per step: all their loads are issued before any store.
  constexpr int HU = WARP_TERMINAL_HANDS_PER_STEP;
  int h = lane;
  for (; h + 32 * (HU - 1) < hpp; h += 32 * HU) {
    R v[HU], f[HU];
#pragma unroll
    for (int u = 0; u < HU; u++) value(h + 32 * u, v[u], f[u]);
#pragma unroll
    for (int u = 0; u < HU; u++) out[h + 32 * u] = v[u];
    if (fout) {
#pragma unroll
      for (int u = 0; u < HU; u++) fout[h + 32 * u] = f[u];
    }
  }
  for (; h < hpp; h += 32) {
    R v0, f0;
    value(h, v0, f0);
    out[h] = v0;
    if (fout) fout[h] = f0;
  }
  __syncwarp();  // the next task overwrites the row and the prefixes
}

}  // namespace dcfr
