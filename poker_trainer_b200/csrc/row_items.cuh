// Per-node row work of a DCFR traversal, shared by the level kernels
// (kernels.cu) and the batched river kernel (batch.cu). Every f32 operation
// is performed in the order of the reference CPU solver
// (AhanDatta/Poker-Trainer crates/solver/src/cfr.rs, river.rs): a thread
// handles 4 hands with 128-bit loads and stores, and all arithmetic is per
// hand.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"

namespace dcfr {

__device__ __forceinline__ float max0(float x) { return x > 0.0f ? x : 0.0f; }

// recip (cfr.rs:114-121): 1/d for a positive d whose reciprocal is finite.
__device__ __forceinline__ float recipf(float d) {
  float i = 1.0f / d;
  return (d > 0.0f && isfinite(i)) ? i : 0.0f;
}

__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float& at(float4& v, int j) { return (&v.x)[j]; }
// Per-player fields of the kernel arguments, selected without indexing the
// parameter arrays (a dynamic index would copy them to local memory).
template <typename T>
__device__ __forceinline__ T pick(int q, const T (&v)[2]) {
  return q ? v[1] : v[0];
}

__device__ __forceinline__ bool nz4(const float4& v) { return v.x != 0.0f || v.y != 0.0f || v.z != 0.0f || v.w != 0.0f; }

// ------------------------------------------------- 16-bit compressed storage
// Storage::Compressed (storage.rs:87-330): per decision node, i16 regrets
// scaled by rscale[slot] / 32767 and u16 strategy sums scaled by
// sscale[slot] / 65535, where the node's scale is the max |value| of its
// block after its last update. Regret matching reads the raw i16 values (a
// positive scale cancels); every update decodes, updates in f32, takes the
// block's new max and re-encodes. A block covers a whole row of the node, so
// the max is a block reduction; every thread of the block must call it.
__device__ __forceinline__ float4 ldq(const int16_t* p) {
  const short4 q = *reinterpret_cast<const short4*>(p);
  return make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
}
__device__ __forceinline__ float4 ldq(const uint16_t* p) {
  const ushort4 q = *reinterpret_cast<const ushort4*>(p);
  return make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
}
__device__ __forceinline__ float4 scale4(float4 v, float s) {
  return make_float4(v.x * s, v.y * s, v.z * s, v.w * s);
}
__device__ __forceinline__ float absmax4(const float4& v) {
  return fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
}
// Regret encoding (storage.rs:284-297): round half away from zero, then
// Rust's saturating `as i16` (truncation toward zero).
__device__ __forceinline__ int16_t enc_regret(float v, float inv) {
  const float y = v * inv;
  const float t = y + copysignf(0.5f, y);
  return t >= 32767.0f ? (int16_t)32767 : t <= -32768.0f ? (int16_t)-32768 : (int16_t)__float2int_rz(t);
}
// Strategy-sum encoding (storage.rs:318-325): max(v, 0) * inv + 0.5,
// saturating `as u16`.
__device__ __forceinline__ uint16_t enc_sum(float v, float inv) {
  const float t = fmaxf(v, 0.0f) * inv + 0.5f;
  return t >= 65535.0f ? (uint16_t)65535 : (uint16_t)__float2uint_rz(t);
}
// Max over the block (all threads call it, in the same order; blockDim a
// multiple of 32). Calls alternate between two scratch rows (`phase`, one
// counter per thread that every thread advances alike), so one barrier per
// call suffices: a row is rewritten only after the next call's barrier,
// which every thread passes after its reads of that row.
__device__ __forceinline__ float block_max(float v, int& phase) {
  __shared__ float red[2][32];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, d));
  float* row = red[phase & 1];
  phase++;
  if ((threadIdx.x & 31) == 0) row[threadIdx.x >> 5] = v;
  __syncthreads();
  float m = 0.0f;
  const int nw = (int)(blockDim.x >> 5);
  for (int w = 0; w < nw; w++) m = fmaxf(m, row[w]);
  return m;
}

// ------------------------------------------------------------- down levels
// Opponent split (cfr.rs:384-420 / river.rs:115-160) and chance split
// (cfr.rs:448-456).
// One warp's item: hands [h0, h0 + 128) of one node, 4 per lane.
// COMP: compressed storage (T.cards holds the node's scale slot); the whole
// block takes part in every call.
template <int MODE, int MAXA, int KIND, bool COMP = false>
__device__ __forceinline__ void down_item(const RowArgs& A, const DownTask& T, int h0, int lane, int* phase = nullptr) {
  const uint32_t live = A.alive[T.in_slot];
  if (live == 0) return;  // dead subtree: children stay dead
  const int o = A.p ^ 1;
  const int hp = pick(o, A.hp);
  const bool valid = h0 < hp;
  const size_t stride = (size_t)A.stride;
  float4 r = valid ? ld4(A.reach + (size_t)T.in_slot * stride + h0) : make_float4(0.f, 0.f, 0.f, 0.f);
  if constexpr (KIND == D_OPP_SPLIT) {
    const int na = (int)T.nchild;
    const float uniform = 1.0f / (float)na;
    float4 x[MAXA];
    float4 inv;
    const float* base = (MODE == M_CFR ? A.regrets : A.sums) + T.store + h0;
    float* sb = A.sums + T.store + h0;
    float4 sums[MODE == M_CFR ? MAXA : 1];
    // Compressed: the sums' decode factor (storage.rs:259-262, 313-314).
    const float sdec = COMP ? A.sscale[T.cards] / 65535.0f : 0.0f;
    // Every storage load of the node is issued before the arithmetic.
    if constexpr (COMP) {
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na) {
          const size_t e = T.store + (size_t)a * hp + h0;
          // CFR: raw i16 regrets (regret matching); otherwise the decoded sums.
          x[a] = !valid ? make_float4(0.f, 0.f, 0.f, 0.f)
                        : (MODE == M_CFR ? ldq(A.rq + e) : scale4(ldq(A.sq + e), sdec));
        }
      if (MODE == M_CFR) {
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na) sums[a] = valid ? scale4(ldq(A.sq + T.store + (size_t)a * hp + h0), sdec)
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    } else {
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na) x[a] = valid ? ld4(base + (size_t)a * hp) : make_float4(0.f, 0.f, 0.f, 0.f);
      if (MODE == M_CFR) {
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na && valid) sums[a] = ld4(sb + (size_t)a * hp);
      }
    }
    if (MODE == M_CFR) {
      // regret_match_into (cfr.rs:161-192).
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        float s = max0(at(x[0], j));
#pragma unroll
        for (int a = 1; a < MAXA; a++)
          if (a < na) s += max0(at(x[a], j));
        at(inv, j) = recipf(s);
      }
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na)
#pragma unroll
          for (int j = 0; j < VEC; j++) at(x[a], j) = at(inv, j) == 0.0f ? uniform : max0(at(x[a], j)) * at(inv, j);
      // Strategy sums s*gamma + sigma (or + sigma*reach) (cfr.rs:395-407).
      const DiscountD d = *A.disc;
      float smax = 0.0f;
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na && valid) {
          float4 s = sums[MODE == M_CFR ? a : 0];
#pragma unroll
          for (int j = 0; j < VEC; j++) {
            float add = d.reach_weighted ? at(x[a], j) * at(r, j) : at(x[a], j);
            at(s, j) = at(s, j) * d.strat + add;
          }
          if constexpr (COMP) {
            sums[MODE == M_CFR ? a : 0] = s;
            smax = fmaxf(smax, absmax4(s));
          } else {
            st4(sb + (size_t)a * hp, s);
          }
        }
      if constexpr (COMP) {
        // The node's new scale and the re-encoded sums (storage.rs:315-328).
        const float mx = block_max(smax, *phase);
        const float sinv = mx > 0.0f ? 65535.0f / mx : 0.0f;
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na && valid) {
            const float4 s = sums[MODE == M_CFR ? a : 0];
            ushort4 q = make_ushort4(0, 0, 0, 0);
            if (mx > 0.0f) q = make_ushort4(enc_sum(s.x, sinv), enc_sum(s.y, sinv), enc_sum(s.z, sinv), enc_sum(s.w, sinv));
            *reinterpret_cast<ushort4*>(A.sq + T.store + (size_t)a * hp + h0) = q;
          }
        if (threadIdx.x == 0) A.sscale[T.cards] = mx;
      }
    } else {
      // normalize_in_place (cfr.rs:124-154).
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        float s = at(x[0], j);
#pragma unroll
        for (int a = 1; a < MAXA; a++)
          if (a < na) s += at(x[a], j);
        at(inv, j) = recipf(s);
      }
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na)
#pragma unroll
          for (int j = 0; j < VEC; j++) at(x[a], j) = at(inv, j) == 0.0f ? uniform : at(x[a], j) * at(inv, j);
    }
    // Child reach = strategy * reach, and child liveness.
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na) {
        float4 c;
#pragma unroll
        for (int j = 0; j < VEC; j++) at(c, j) = at(x[a], j) * at(r, j);
        if (valid) st4(A.reach + (size_t)(T.out_slot + a) * stride + h0, c);
        bool any = __any_sync(0xffffffffu, valid && nz4(c));
        if (any && lane == 0) A.alive[T.out_slot + a] = 1u;
      }
  } else {
    // Chance split: reach*factor, opponent hands holding the card zeroed.
    uchar4 oc1 = make_uchar4(255, 255, 255, 255), oc2 = oc1;
    if (valid) {
      oc1 = *reinterpret_cast<const uchar4*>(pick(o, A.hc1) + h0);
      oc2 = *reinterpret_cast<const uchar4*>(pick(o, A.hc2) + h0);
    }
    const uint8_t* cards = A.chance_cards + T.cards;
    for (uint32_t i = 0; i < T.nchild; i++) {
      const uint8_t card = cards[i];
      float4 c;
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        uint8_t a1 = (&oc1.x)[j], a2 = (&oc2.x)[j];
        at(c, j) = (a1 == card || a2 == card) ? 0.0f : at(r, j) * T.factor;
      }
      if (valid) st4(A.reach + (size_t)(T.out_slot + i) * stride + h0, c);
      bool any = __any_sync(0xffffffffu, valid && nz4(c));
      if (any && lane == 0) A.alive[T.out_slot + i] = 1u;
    }
  }
}

// --------------------------------------------------------------- up levels
// Traverser node (own_node_update, cfr.rs:315-382), opponent node sum
// (cfr.rs:421-432, river.rs:264-271) and chance sum (cfr.rs:462-478).
// COMP: compressed storage (T.cards holds a traverser node's scale slot);
// the whole block takes part in every call.
template <int MODE, int MAXA, int KIND, bool COMP = false>
__device__ __forceinline__ void up_item(const RowArgs& A, const UpTask& T, int h0, int* phase = nullptr) {
  const uint32_t live = A.alive[T.slot];
  if (live == 0) return;
  const int p = A.p;
  const int hp = pick(p, A.hp);
  if constexpr (COMP && KIND == U_OWN && MODE == M_CFR) {
    // Compressed regret update (storage.rs:272-303 around
    // own_node_update, cfr.rs:347-379): every thread reaches the block max.
    const bool valid = h0 < hp;
    const size_t stride = (size_t)A.stride;
    const int na = (int)T.nchild;
    const float rdec = A.rscale[T.cards] / 32767.0f;
    float4 cfv[MAXA], r[MAXA];
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na) {
        cfv[a] = valid ? ld4(A.vals + (size_t)(T.child + a) * stride + h0) : z;
        r[a] = valid ? scale4(ldq(A.rq + T.store + (size_t)a * hp + h0), rdec) : z;
      }
    const DiscountD d = *A.disc;
    float4 out;
#pragma unroll
    for (int j = 0; j < VEC; j++) {
      float s = max0(at(r[0], j));
#pragma unroll
      for (int a = 1; a < MAXA; a++)
        if (a < na) s += max0(at(r[a], j));
      float o = 0.0f;
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na) o += max0(at(r[a], j)) * at(cfv[a], j);
      float iv = recipf(s);
      o *= iv;
      if (iv == 0.0f) {
        float m = -0.0f;
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na) m += at(cfv[a], j);
        o = m * (1.0f / (float)na);
      }
      at(out, j) = o;
    }
    float rmax = 0.0f;
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na) {
#pragma unroll
        for (int j = 0; j < VEC; j++) {
          float x = at(r[a], j);
          float disc = x > 0.0f ? d.pos : d.neg;
          at(r[a], j) = x * disc + at(cfv[a], j) - at(out, j);
        }
        if (valid) rmax = fmaxf(rmax, absmax4(r[a]));
      }
    const float mx = block_max(rmax, *phase);
    const float rinv = mx > 0.0f ? 32767.0f / mx : 0.0f;
    if (valid) {
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na) {
          short4 q = make_short4(0, 0, 0, 0);
          if (mx > 0.0f)
            q = make_short4(enc_regret(r[a].x, rinv), enc_regret(r[a].y, rinv), enc_regret(r[a].z, rinv),
                            enc_regret(r[a].w, rinv));
          *reinterpret_cast<short4*>(A.rq + T.store + (size_t)a * hp + h0) = q;
        }
      st4(A.vals + (size_t)T.node * stride + h0, out);
    }
    if (threadIdx.x == 0) A.rscale[T.cards] = mx;
    return;
  }
  if (h0 >= hp) return;
  const size_t stride = (size_t)A.stride;
  float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
  if constexpr (KIND == U_OWN) {
    const int na = (int)T.nchild;
    float4 cfv[MAXA];
    // Child values and the node's storage block (regrets in CFR, strategy
    // sums in Average mode) are loaded together.
    float4 st[MODE == M_BR ? 1 : MAXA];
    const float* sbase = (MODE == M_CFR ? A.regrets : A.sums) + T.store + h0;
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na) cfv[a] = ld4(A.vals + (size_t)(T.child + a) * stride + h0);
    if (MODE != M_BR) {
      if constexpr (COMP) {
        // Average mode: the decoded strategy sums (the CFR update is above).
        const float sdec = A.sscale[T.cards] / 65535.0f;
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na) st[MODE == M_BR ? 0 : a] = scale4(ldq(A.sq + T.store + (size_t)a * hp + h0), sdec);
      } else {
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na) st[MODE == M_BR ? 0 : a] = ld4(sbase + (size_t)a * hp);
      }
    }
    if (MODE == M_BR) {
      out = cfv[0];
#pragma unroll
      for (int a = 1; a < MAXA; a++)
        if (a < na)
#pragma unroll
          for (int j = 0; j < VEC; j++) at(out, j) = at(cfv[a], j) > at(out, j) ? at(cfv[a], j) : at(out, j);
    } else if (MODE == M_AVG) {
      float4* s = st;
      float4 inv;
      const float uniform = 1.0f / (float)na;
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        float d = at(s[0], j);
#pragma unroll
        for (int a = 1; a < MAXA; a++)
          if (a < na) d += at(s[a], j);
        at(inv, j) = recipf(d);
      }
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na)
#pragma unroll
          for (int j = 0; j < VEC; j++) {
            float sv = at(inv, j) == 0.0f ? uniform : at(s[a], j) * at(inv, j);
            at(out, j) += sv * at(cfv[a], j);
          }
    } else {
      const DiscountD d = *A.disc;
      float4* r = st;
      float4 inv;
      float* rb = A.regrets + T.store + h0;
#pragma unroll
      for (int j = 0; j < VEC; j++) {
        float s = max0(at(r[0], j));
#pragma unroll
        for (int a = 1; a < MAXA; a++)
          if (a < na) s += max0(at(r[a], j));
        float o = 0.0f;
#pragma unroll
        for (int a = 0; a < MAXA; a++)
          if (a < na) o += max0(at(r[a], j)) * at(cfv[a], j);
        float iv = recipf(s);
        o *= iv;
        if (iv == 0.0f) {
          float m = -0.0f;
#pragma unroll
          for (int a = 0; a < MAXA; a++)
            if (a < na) m += at(cfv[a], j);
          o = m * (1.0f / (float)na);
        }
        at(out, j) = o;
        at(inv, j) = iv;
      }
      (void)inv;
#pragma unroll
      for (int a = 0; a < MAXA; a++)
        if (a < na) {
#pragma unroll
          for (int j = 0; j < VEC; j++) {
            float x = at(r[a], j);
            float disc = x > 0.0f ? d.pos : d.neg;
            at(r[a], j) = x * disc + at(cfv[a], j) - at(out, j);
          }
          st4(rb + (size_t)a * hp, r[a]);
        }
    }
  } else if constexpr (KIND == U_OPP_SUM) {
    // Loads first (independent), then the sum in child order.
    const int na = (int)T.nchild;
    float4 v[MAXA];
    bool clive[MAXA];
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na) {
        clive[a] = A.alive[T.child_slot + a] != 0;
        v[a] = ld4(A.vals + (size_t)(T.child + a) * stride + h0);
      }
#pragma unroll
    for (int a = 0; a < MAXA; a++)
      if (a < na && clive[a])
#pragma unroll
        for (int j = 0; j < VEC; j++) at(out, j) += at(v[a], j);
  } else {
    double acc[VEC] = {0.0, 0.0, 0.0, 0.0};
    const uint8_t* hc1p = pick(p, A.hc1);
    const uint8_t* hc2p = pick(p, A.hc2);
    const uchar4 mc1 = *reinterpret_cast<const uchar4*>(hc1p + h0);
    const uchar4 mc2 = *reinterpret_cast<const uchar4*>(hc2p + h0);
    const uint8_t* cards = A.chance_cards + T.cards;
    // Children in batches: flags, cards and rows are loaded before the f64
    // sum, which stays in card order.
    constexpr int B = 8;
    for (uint32_t i0 = 0; i0 < T.nchild; i0 += B) {
      bool live[B];
      uint8_t card[B];
      float4 v[B];
#pragma unroll
      for (int k = 0; k < B; k++) {
        const uint32_t i = i0 + k;
        live[k] = i < T.nchild && A.alive[T.child_slot + i] != 0;
        card[k] = i < T.nchild ? cards[i] : 255;
      }
#pragma unroll
      for (int k = 0; k < B; k++)
        if (live[k]) v[k] = ld4(A.vals + (size_t)(T.child + i0 + k) * stride + h0);
#pragma unroll
      for (int k = 0; k < B; k++)
        if (live[k])
#pragma unroll
          for (int j = 0; j < VEC; j++) {
            bool blocked = (&mc1.x)[j] == card[k] || (&mc2.x)[j] == card[k];
            acc[j] += blocked ? 0.0 : (double)at(v[k], j);
          }
    }
    constexpr int BI = 4;
    const int np = pick(p, A.n);
    for (uint32_t k0 = 0; k0 < T.iso_count; k0 += BI) {
      bool live[BI];
      float x[BI][VEC];
      bool blk[BI][VEC];
#pragma unroll
      for (int k = 0; k < BI; k++) {
        live[k] = false;
        if (k0 + k < T.iso_count) {
          const IsoRefD ref = A.iso[T.iso_first + k0 + k];
          live[k] = A.alive[T.child_slot + ref.ci] != 0;
          const uint8_t card = cards[ref.ci];
          const float* row = A.vals + (size_t)(T.child + ref.ci) * stride;
          const uint16_t* perm = A.perm + (size_t)(p * 6 + ref.pair) * stride;
#pragma unroll
          for (int j = 0; j < VEC; j++) {
            x[k][j] = 0.0f;
            blk[k][j] = true;
            const int h = h0 + j;
            if (h < np) {
              const int q = perm[h];
              blk[k][j] = hc1p[q] == card || hc2p[q] == card;
              x[k][j] = row[q];
            }
          }
        }
      }
#pragma unroll
      for (int k = 0; k < BI; k++)
        if (live[k])
#pragma unroll
          for (int j = 0; j < VEC; j++)
            if (h0 + j < np) acc[j] += blk[k][j] ? 0.0 : (double)x[k][j];
    }
#pragma unroll
    for (int j = 0; j < VEC; j++) at(out, j) = (float)acc[j];
  }
  st4(A.vals + (size_t)T.node * stride + h0, out);
}

}  // namespace dcfr
