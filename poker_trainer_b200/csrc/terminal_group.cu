// Group-per-terminal evaluation: the fixed-point prefix sums of
// warp_terminal_task (warp_terminal.cuh) with every terminal evaluated by a
// group of GROUP_WARPS warps instead of one.
//
// The warp-per-terminal kernel keeps one terminal in flight per warp, and
// each terminal needs its own prefix array (8 bytes per layout element) and
// two reach rows in shared memory, so at about 470 hands only 14 warps fit on
// an SM and the kernel is bound by latency (a third of the issue slots used).
// A group of two warps shares one terminal's prefix array and rows: the same
// number of terminals in flight, twice the warps, half the serial work per
// warp. The warps of a group meet at named barriers (one id per group), three
// per showdown and two per fold:
//   (1) the row has landed and each warp has published the maximum of the
//       entries it copied itself;
//   (2) each warp has published the total of its part of the scan (a fold:
//       its part of the total and the card totals);
//   (3) the prefixes and each card segment's start and end prefixes are
//       written (by the threads whose elements hold the boundaries).
// The next task's row is requested after barrier (1), when every warp of the
// group is done with the previous task and its row buffer.
//
// The values are bit-identical to warp_terminal_task's: the same integer
// sums, the same conversions and the same rounding order per terminal kind.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "warp_terminal.cuh"

namespace dcfr {

constexpr int GROUP_WARPS = 2;
constexpr int GROUP_THREADS = 32 * GROUP_WARPS;
// Groups per block (named barriers 1..GROUP_MAX). Twelve leave 80 registers a
// thread with no spills; fourteen (72 registers, a few spills) measured 1.5%
// slower on the flop.
constexpr int GROUP_MAX = 12;

// Shared memory of a block: the staged layout (shared by the block's
// groups), then per group two reach rows, the prefix array, the card-segment
// start and end prefixes (16 bytes per card) and the warps' partial results.
struct GroupSmem {
  size_t same, cat, rec, seg, group0, row_bytes, g_off, cst_off, red_off, group_bytes, total;
  __host__ __device__ GroupSmem(int stride, int cstride, int tstride, int groups) {
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    same = 0;
    cat = up16(same + (size_t)stride * 2);
    rec = up16(cat + (size_t)cstride * 2);
    seg = up16(rec + (size_t)tstride * 16);
    group0 = up16(seg + FAST_SEGS * 2);
    row_bytes = up16((size_t)stride * 4);
    g_off = 2 * row_bytes;
    // Prefixes 0..L (L <= cstride); a fold keeps its 52 card totals here.
    const size_t gn = (size_t)cstride + 2 > 56 ? (size_t)cstride + 2 : 56;
    cst_off = g_off + up16(gn * 8);
    red_off = cst_off + up16(52 * 16);
    group_bytes = red_off + up16((size_t)GROUP_WARPS * 12);
    total = group0 + (size_t)groups * group_bytes;
  }
};

__device__ __forceinline__ void group_sync(int id) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "n"(GROUP_THREADS) : "memory");
}

// The group's threads copy the row of `slot` in 16-byte chunks: thread gt
// takes chunks gt, gt + GROUP_THREADS, ... (the same chunks it reads back
// for its part of the row maximum).
__device__ __forceinline__ void group_row_prefetch(const FastArgs& A, uint32_t slot, float* row, int gt) {
  const int hpo = (A.p ^ 1) ? A.hp[1] : A.hp[0];
  const char* src = reinterpret_cast<const char*>(A.reach + (size_t)slot * A.stride);
  const uint32_t dst = (uint32_t)__cvta_generic_to_shared(row);
  for (int i = gt; i < hpo / 4; i += GROUP_THREADS)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + 16u * (uint32_t)i), "l"(src + 16 * (size_t)i)
                 : "memory");
}

// One terminal task evaluated by the GROUP_THREADS threads of a group (gt
// = thread in the group). row: the group's copy of the task's reach row, its
// own chunks waited for by every thread. next_slot / next_row: the row to
// request after barrier (1) (NONE32: none). bfirst: the first segment
// boundary b >= 1 with seg[b] >= this thread's first scan element.
__device__ __forceinline__ void group_task(const FastArgs& A, const FastTask& T, const WarpLayout& Y, const float* row,
                                           long long* G, long long* cst, long long* gsum, float* gmax, int gt, int bar,
                                           int bfirst, uint32_t next_slot, float* next_row) {
  const int lane = gt & 31, w = gt >> 5;
  const int p = A.p, o = p ^ 1;
  const int hpo = o ? A.hp[1] : A.hp[0], hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  const int L = Y.L;
  // 1. Row maximum: each thread's own copied chunks, then the group's.
  float mx = 0.0f;
  for (int i = gt; i < hpo / 4; i += GROUP_THREADS) {
    const float4 v = reinterpret_cast<const float4*>(row)[i];
    mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, d));
  if (lane == 0) gmax[w] = mx;
  group_sync(bar);  // (1)
  if (next_slot != NONE32) group_row_prefetch(A, next_slot, next_row, gt);
  cp_async_commit();
#pragma unroll
  for (int k = 0; k < GROUP_WARPS; k++) mx = fmaxf(mx, gmax[k]);
  const int S = scale_exponent(mx);
  const double scale = pow2(S), inv = pow2(-S);
  const double pa = T.a * inv, pb = T.b * inv, pc = T.c * inv, pd = T.d * inv;
  const uint32_t kind = T.kind;
  const bool fold = kind == T_FOLD_SCALAR || kind == T_FOLD_BATCH;
  const bool scalar = kind == T_FOLD_SCALAR || kind == T_SHOWDOWN_SCALAR;
  float* out = A.vals + (size_t)T.row * A.stride;
  if (fold) {
    // eval_fold (eval.rs:40-64): the total and each card's total.
    long long t0 = 0;
    for (int k = gt; k < Y.seg[1]; k += GROUP_THREADS) t0 += fixed(row[Y.cat[k]], scale);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) t0 += __shfl_xor_sync(0xffffffffu, t0, d);
    if (lane == 0) gsum[w] = t0;
    for (int c = gt; c < 52; c += GROUP_THREADS) {
      long long tc = 0;
      for (int k = Y.seg[1 + c]; k < Y.seg[2 + c]; k++) tc += fixed(row[Y.cat[k]], scale);
      G[c] = tc;
    }
    group_sync(bar);  // (2)
    t0 = 0;
#pragma unroll
    for (int k = 0; k < GROUP_WARPS; k++) t0 += gsum[k];
    for (int h = gt; h < hpp; h += GROUP_THREADS) {
      float v = 0.0f;
      if (h < np) {
        const uint32_t q = Y.rec[h].w;
        const int a = (int)(q & 0xFF), b = (int)((q >> 8) & 0xFF);
        const uint16_t sm = Y.same[h];
        const long long si = sm == 0xFFFF ? 0ll : fixed(row[sm], scale);
        const long long F = t0 - G[a] - G[b] + si;
        v = (scalar && t0 == 0) ? 0.0f : (float)(pa * (double)F);
      }
      out[h] = v;
    }
    return;
  }
  // 2. Elements in layout order: E consecutive elements per thread.
  const int E = ((L + GROUP_THREADS - 1) / GROUP_THREADS) | 1;
  const int k0 = gt * E, k1 = min(L, k0 + E);
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
  if (lane == 31) gsum[w] = inc;
  group_sync(bar);  // (2)
  long long acc = inc - local, total = 0;
#pragma unroll
  for (int q = 0; q < GROUP_WARPS; q++) {
    if (q < w) acc += gsum[q];
    total += gsum[q];
  }
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
  // Segment boundaries inside this thread's elements (its own prefixes);
  // those at the layout's end (empty trailing segments, and boundary 53)
  // are the total.
  // Boundary b (1..53) starts card b - 1's segment and ends card b - 2's:
  // cpair[c] = {start, end} of card c, one 16-byte read per card.
  auto put = [&](int b, long long v) {
    if (b <= 52) cst[2 * (b - 1)] = v;
    if (b >= 2) cst[2 * (b - 2) + 1] = v;
  };
  for (int b = bfirst; b < FAST_SEGS && Y.seg[b] < k1; b++) put(b, G[Y.seg[b]]);
  if (gt == 0) {
    G[L] = total;  // a card segment's end can be the layout's end
    for (int b = FAST_SEGS - 1; b >= 1 && Y.seg[b] >= L; b--) put(b, total);
  }
  group_sync(bar);  // (3)

  // 3. Values in hand order. Boundary 1 closes the strength segment, so T0
  // is card 0's start.
  const longlong2* cpair = reinterpret_cast<const longlong2*>(cst);
  const long long T0 = cst[0];
  float* fout = T.frow != NONE32 ? A.vals + (size_t)T.frow * A.stride : nullptr;
  auto value = [&](int h, float& v, float& fv) {
    v = 0.0f;
    fv = 0.0f;
    if (h >= np) return;
    const uint4 q = Y.rec[h];
    const int a = (int)(q.w & 0xFF), b = (int)((q.w >> 8) & 0xFF);
    const longlong2 pa2 = cpair[a], pb2 = cpair[b];
    const long long sa = pa2.x, ea = pa2.y, sb = pb2.x, eb = pb2.y;
    const uint16_t sm = Y.same[h];
    const long long si = sm == 0xFFFF ? 0ll : fixed(row[sm], scale);
    const longlong2 ca = make_longlong2(sa, ea - sa), cb = make_longlong2(sb, eb - sb);
    const long long F = T0 - ca.y - cb.y + si;
    if (q.w >> 16) {
      const long long Gw = G[q.x & 0xFFFF], Gs = G[q.x >> 16];
      const long long Gaw = G[q.y & 0xFFFF], Gas = G[q.y >> 16];
      const long long Gbw = G[q.z & 0xFFFF], Gbs = G[q.z >> 16];
      const long long Wn = (Gw + ca.x + cb.x) - Gaw - Gbw;
      const long long Lx = (T0 + Gas + Gbs) - Gs - (ca.x + ca.y) - (cb.x + cb.y);
      if (scalar) {
        v = (float)(pa * (double)Wn) + (float)(pb * (double)Lx);
      } else {
        double res = pa * (double)Wn;
        res += pb * (double)Lx;
        v = (float)res;
      }
      if (T.c != 0.0) {
        const long long eq = (Gs - Gw) - (Gas - Gaw) - (Gbs - Gbw) + si;
        v += (float)(pc * (double)eq);
      }
    }
    if (fout) fv = (float)(pd * (double)F);
  };
  // Two hands per step: both hands' loads are issued before the stores.
  int h = gt;
  for (; h + GROUP_THREADS < hpp; h += 2 * GROUP_THREADS) {
    float v0, f0, v1, f1;
    value(h, v0, f0);
    value(h + GROUP_THREADS, v1, f1);
    out[h] = v0;
    out[h + GROUP_THREADS] = v1;
    if (fout) {
      fout[h] = f0;
      fout[h + GROUP_THREADS] = f1;
    }
  }
  for (; h < hpp; h += GROUP_THREADS) {
    float v0, f0;
    value(h, v0, f0);
    out[h] = v0;
    if (fout) fout[h] = f0;
  }
}

// Block b takes the contiguous task range [b N / B, (b+1) N / B) of the N
// layout-ordered tasks; its groups take the range's tasks in turn (group g:
// tasks g, g + NG, ...). The block stages a unit's layout (a maximal run of
// tasks on one layout) once, with a block barrier only where its range
// crosses from one unit to the next.
__global__ void __launch_bounds__(GROUP_THREADS* GROUP_MAX, 1)
    group_terminal_kernel(FastArgs A, const FastTask* __restrict__ tasks, const TermUnit* __restrict__ units,
                          int nunits, int ntasks) {
  extern __shared__ __align__(16) unsigned char smem_g[];
  const int NG = (int)blockDim.x / GROUP_THREADS;
  const GroupSmem L_(A.stride, A.cstride, A.tstride, NG);
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_g + L_.same);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_g + L_.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_g + L_.rec);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_g + L_.seg);
  const int tid = threadIdx.x, grp = tid / GROUP_THREADS, gt = tid - grp * GROUP_THREADS;
  unsigned char* gb = smem_g + L_.group0 + (size_t)grp * L_.group_bytes;
  float* const row_a = reinterpret_cast<float*>(gb);
  float* const row_b = reinterpret_cast<float*>(gb + L_.row_bytes);
  long long* G = reinterpret_cast<long long*>(gb + L_.g_off);
  long long* cst = reinterpret_cast<long long*>(gb + L_.cst_off);
  long long* gsum = reinterpret_cast<long long*>(gb + L_.red_off);
  float* gmax = reinterpret_cast<float*>(gb + L_.red_off + GROUP_WARPS * 8);
  const int bar = 1 + grp;

  const int p = A.p;
  const int hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  for (int h = tid; h < hpp; h += blockDim.x) {
    const uint32_t sm = h < np ? A.same[h] : NONE32;
    ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
  }
  const int t0 = (int)(((long long)blockIdx.x * ntasks) / gridDim.x);
  const int t1 = (int)(((long long)(blockIdx.x + 1) * ntasks) / gridDim.x);
  int u = 0;
  {
    int hi = nunits - 1;
    while (u < hi) {
      const int mid = (u + hi) >> 1;
      if ((int)(units[mid].first + units[mid].count) <= t0) u = mid + 1;
      else hi = mid;
    }
  }
  int buf = 0;
  int next = t0 + grp;  // this group's current task
  bool live = false;
  if (next < t1) {
    live = A.alive[tasks[next].slot] != 0;
    if (live) group_row_prefetch(A, tasks[next].slot, row_a, gt);
  }
  cp_async_commit();
  for (; u < nunits && (int)units[u].first < t1; u++) {
    const TermUnit U = units[u];
    __syncthreads();  // the previous unit's groups are done with the layout
    const size_t lay = (size_t)U.layout * 2 + p;
    const uint16_t* gseg = A.seg + lay * FAST_SEGS;
    if (tid < FAST_SEGS) sseg[tid] = gseg[tid];
    const int L = gseg[FAST_SEGS - 1];
    const uint16_t* gcat = A.cat + lay * A.cstride;
    for (int k = tid; k < L; k += blockDim.x) scat[k] = gcat[k];
    const uint4* grec = A.rec + lay * A.tstride;
    for (int h = tid; h < np; h += blockDim.x) srec[h] = grec[h];
    __syncthreads();
    const WarpLayout Y{ssame, scat, srec, sseg, L};
    // This thread's first segment boundary at or after its first element.
    const int k0 = gt * (((L + GROUP_THREADS - 1) / GROUP_THREADS) | 1);
    int bfirst = 1;
    while (bfirst < FAST_SEGS && sseg[bfirst] < k0) bfirst++;
    const int end = min(t1, (int)(U.first + U.count));
    for (; next < end; next += NG) {
      cp_async_wait<0>();  // this task's row (own copies)
      const int nx = next + NG;
      const bool nlive = nx < t1 && A.alive[tasks[nx].slot] != 0;
      float* const cur_row = buf ? row_b : row_a;
      float* const nxt_row = buf ? row_a : row_b;
      // Dead subtree (cfr.rs:267-274): row untouched.
      if (live) {
        group_task(A, tasks[next], Y, cur_row, G, cst, gsum, gmax, gt, bar, bfirst,
                   nlive ? tasks[nx].slot : NONE32, nxt_row);
      } else {
        // The group's other warps may still read the previous task's row
        // from the buffer the next row goes to.
        if (nlive) {
          group_sync(bar);
          group_row_prefetch(A, tasks[nx].slot, nxt_row, gt);
        }
        cp_async_commit();
      }
      live = nlive;
      buf ^= 1;
    }
  }
  cp_async_wait<0>();
}

size_t group_terminal_smem(int stride, int cstride, int tstride, int groups) {
  return GroupSmem(stride, cstride, tstride, groups).total;
}

// Groups per block (1..GROUP_MAX) that maximise resident groups per SM, and
// the blocks per SM at that count; 0 if none fits.
int group_terminal_setup(int stride, int cstride, int tstride, int& blocks_per_sm) {
  int dev = 0, optin = 0;
  blocks_per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  const void* fn = (const void*)group_terminal_kernel;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess) return 0;
  int best_g = 0, best_b = 0;
  for (int g = 1; g <= GROUP_MAX; g++) {
    const size_t smem = group_terminal_smem(stride, cstride, tstride, g);
    if (smem > (size_t)optin) break;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, g * GROUP_THREADS, smem) != cudaSuccess) return 0;
    if (b > 0 && g * b >= best_g * best_b) {
      best_g = g;
      best_b = b;
    }
  }
  blocks_per_sm = best_b;
  return best_g;
}

void launch_group_terminal(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                           int groups, int max_blocks, cudaStream_t s) {
  if (nunits <= 0 || ntasks <= 0) return;
  // At most one block per task: every block's range is non-empty.
  const int blocks = ntasks < max_blocks ? ntasks : max_blocks;
  const size_t smem = group_terminal_smem(A.stride, A.cstride, A.tstride, groups);
  group_terminal_kernel<<<blocks, groups * GROUP_THREADS, smem, s>>>(A, tasks, units, nunits, ntasks);
}

}  // namespace dcfr
