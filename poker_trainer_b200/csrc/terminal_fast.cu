// Fast-precision terminal evaluation: the counterpart of the reference's
// default GPU precision, GpuPrecision::Fast (crates/solver/src/gpu/mod.rs:53-58),
// which agrees with the exact evaluators except for rare one-rounding-step
// differences.
//
// The exact evaluators (crates/solver/src/eval.rs:40-379) sweep the opponent's
// strength-sorted reach and accumulate f64 sums in a fixed order. Here every
// f32 reach value of a row is first converted to a 64-bit fixed-point integer
// (scaled by a power of two chosen from the row's maximum so the row's sum
// stays below 2^62); integer sums are exact and associative, so one
// block-wide prefix scan over the layout of terminal_fast.cu's segments gives
// every sum the evaluators need as a difference of two prefixes:
//   weaker (win)   = G[w] - (blocked by card a) - (blocked by card b)
//   stronger (lose)= (T - G[s]) - (card a's stronger part) - (card b's)
//   equal (tie)    = (G[s] - G[w]) - ... + identical hand   (eval.rs:347-379)
//   fold           = T - (card a total) - (card b total) + identical hand
// Each integer result is converted to f64 once, scaled back, multiplied by the
// payoff and rounded to f32 in the evaluator's own combination order
// (scalar: eval_showdown's two f32 parts; batched: showdown_batch's f64 sum).
// Fixed point drops reach below 2^-51 of the row maximum, far below f64's
// rounding of the reference's sums, so the f32 results match except where the
// reference's own rounding lands next to an f32 boundary.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "warp_terminal.cuh"

namespace dcfr {


// One thread per (layout, traverser): layouts 0..nboards-1 are the showdown
// boards' strength tables, layout nboards lists the opponent's hands in hand
// order for fold terminals.
__global__ void fast_layout_kernel(const EntryD* __restrict__ tables, const uint32_t* __restrict__ count, int tstride,
                                   int nboards, const uint8_t* hc1_0, const uint8_t* hc2_0, const uint8_t* hc1_1,
                                   const uint8_t* hc2_1, int n0, int n1, uint16_t* cat, uint16_t* seg, uint4* rec,
                                   int cstride) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= (nboards + 1) * 2) return;
  const int b = id >> 1, p = id & 1, o = p ^ 1;
  const uint8_t* mc1 = p ? hc1_1 : hc1_0;
  const uint8_t* mc2 = p ? hc2_1 : hc2_0;
  const uint8_t* tc1 = o ? hc1_1 : hc1_0;
  const uint8_t* tc2 = o ? hc2_1 : hc2_0;
  const int np = p ? n1 : n0, no = o ? n1 : n0;
  const bool fold = b == nboards;
  const EntryD* theirs = fold ? nullptr : tables + ((size_t)b * 2 + o) * tstride;
  const EntryD* mine = fold ? nullptr : tables + ((size_t)b * 2 + p) * tstride;
  const int ct = fold ? no : (int)count[(size_t)b * 2 + o];
  const int cm = fold ? 0 : (int)count[(size_t)b * 2 + p];
  uint16_t* C = cat + (size_t)id * cstride;
  uint16_t* S = seg + (size_t)id * FAST_SEGS;
  uint4* R = rec + (size_t)id * tstride;
  auto idx = [&](int j) -> int { return fold ? j : (int)theirs[j].idx; };
  auto card1 = [&](int j) -> int { return fold ? (int)tc1[j] : (int)theirs[j].c1; };
  auto card2 = [&](int j) -> int { return fold ? (int)tc2[j] : (int)theirs[j].c2; };

  int cnt[52], fill[52];
  for (int c = 0; c < 52; c++) cnt[c] = fill[c] = 0;
  for (int j = 0; j < ct; j++) {
    cnt[card1(j)]++;
    cnt[card2(j)]++;
  }
  S[0] = 0;
  int pos = ct;
  for (int c = 0; c < 52; c++) {
    S[1 + c] = (uint16_t)pos;
    pos += cnt[c];
  }
  S[53] = (uint16_t)pos;
  for (int j = 0; j < ct; j++) {
    C[j] = (uint16_t)idx(j);
    const int a = card1(j), bb = card2(j);
    C[S[1 + a] + fill[a]++] = (uint16_t)idx(j);
    C[S[1 + bb] + fill[bb]++] = (uint16_t)idx(j);
  }
  for (int h = 0; h < np; h++) R[h] = make_uint4(0u, 0u, 0u, (uint32_t)mc1[h] | (uint32_t)mc2[h] << 8);
  if (fold) return;
  // Boundaries per strength group of the traverser's table: opponent hands
  // strictly weaker (j, cw) and not stronger (j2, cle).
  int cw[52], cle[52];
  for (int c = 0; c < 52; c++) cw[c] = cle[c] = 0;
  int i = 0, j = 0, j2 = 0;
  while (i < cm) {
    const uint32_t s = mine[i].strength;
    while (j < ct && theirs[j].strength < s) {
      cw[theirs[j].c1]++;
      cw[theirs[j].c2]++;
      j++;
    }
    while (j2 < ct && theirs[j2].strength <= s) {
      cle[theirs[j2].c1]++;
      cle[theirs[j2].c2]++;
      j2++;
    }
    while (i < cm && mine[i].strength == s) {
      const EntryD e = mine[i];
      const int a = e.c1, bb = e.c2;
      R[e.idx] = make_uint4((uint32_t)j | (uint32_t)j2 << 16,
                            (uint32_t)(S[1 + a] + cw[a]) | (uint32_t)(S[1 + a] + cle[a]) << 16,
                            (uint32_t)(S[1 + bb] + cw[bb]) | (uint32_t)(S[1 + bb] + cle[bb]) << 16,
                            (uint32_t)a | (uint32_t)bb << 8 | 1u << 16);
      i++;
    }
  }
}

// Shared-memory layout of a block (all offsets 16-byte aligned); rsize is
// the byte size of a row entry (4 for float rows, 8 for double rows).
struct FastSmem {
  size_t rbuf, g, wsum, fred, cat, rec, same, seg, total;
  __host__ __device__ FastSmem(int stride, int emax, int cstride, int tstride, int rsize = 4) {
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t gn = (size_t)FAST_THREADS * emax + 2;
    rbuf = 0;
    g = up16(rbuf + 2 * (size_t)stride * rsize);
    wsum = up16(g + gn * 8);
    fred = up16(wsum + (FAST_THREADS / 32) * 8);
    cat = up16(fred + 2 * (FAST_THREADS / 32) * rsize);
    rec = up16(cat + (size_t)cstride * 2);
    same = up16(rec + (size_t)tstride * 16);
    seg = up16(same + (size_t)stride * 2);
    total = up16(seg + FAST_SEGS * 2);
  }
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Each block takes a contiguous range of the (board-sorted) task list. The
// board's layout (elements, segment starts, per-hand records) is staged in
// shared memory when the board changes, and the next task's reach row is
// copied in (cp.async) while the current one is evaluated. E (elements per
// thread of the scan, odd) is a compile-time constant so a thread's elements
// stay in registers between the two passes of the scan. R is the row type:
// float for the solve, double for the FP64 best-response oracle (br64.cu),
// whose values are formed in double with no rounding to f32.
//
// DYN: instead of one contiguous range per block, blocks claim chunks of
// FAST_DYN_CHUNK consecutive tasks from `counter` (zeroed before the launch),
// so blocks whose tasks are cheap (dead subtrees are skipped) take more.
// A block claims its next chunk while it starts the current one, so the
// next task's row can still be prefetched across the chunk boundary.
constexpr int FAST_DYN_CHUNK = 8;

template <int E, typename R, bool DYN = false>
__global__ void __launch_bounds__(FAST_THREADS) fast_terminal_kernel(FastArgsT<R> A, const FastTask* __restrict__ tasks,
                                                                     int ntasks, uint32_t* __restrict__ counter = nullptr) {
  extern __shared__ __align__(16) unsigned char smem_fast[];
  constexpr bool F64 = sizeof(R) == 8;
  constexpr int PER16 = 16 / (int)sizeof(R);  // row entries per 16-byte copy
  const FastSmem L_(A.stride, E, A.cstride, A.tstride, (int)sizeof(R));
  R* rbuf = reinterpret_cast<R*>(smem_fast + L_.rbuf);
  long long* G = reinterpret_cast<long long*>(smem_fast + L_.g);
  long long* wsum = reinterpret_cast<long long*>(smem_fast + L_.wsum);
  R* fred = reinterpret_cast<R*>(smem_fast + L_.fred);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_fast + L_.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_fast + L_.rec);
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_fast + L_.same);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_fast + L_.seg);

  const int p = A.p, o = p ^ 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int hpo = o ? A.hp[1] : A.hp[0], hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  __shared__ int s_claim[2];  // DYN: the first chunk, then the chunk after the current one
  int t0, t1;
  if constexpr (DYN) {
    if (tid == 0) s_claim[0] = (int)atomicAdd(counter, (uint32_t)FAST_DYN_CHUNK);
    __syncthreads();
    t0 = s_claim[0];
    t1 = ntasks;
  } else {
    const int per = (ntasks + gridDim.x - 1) / gridDim.x;
    t0 = blockIdx.x * per;
    t1 = min(ntasks, t0 + per);
  }
  if (t0 >= t1) return;
  int cbeg = t0, cend = min(t1, t0 + FAST_DYN_CHUNK), claimed = t1;  // DYN: current chunk, next chunk

  for (int h = tid; h < hpp; h += FAST_THREADS) {
    const uint32_t sm = h < np ? A.same[h] : NONE32;
    ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
  }
  auto prefetch = [&](int ti, int buf) {
    const R* src = A.reach + (size_t)tasks[ti].slot * A.stride;
    R* dst = rbuf + (size_t)buf * A.stride;
    for (int i = tid; i < hpo / PER16; i += FAST_THREADS) cp_async16(dst + PER16 * i, src + PER16 * i);
    cp_async_commit();
  };
  prefetch(t0, 0);
  uint32_t board = NONE32;
  int L = 0;
  FastTask T = tasks[t0];

  // Three block barriers per terminal: after the row maxima (1), after the
  // scan's warp totals (2) and after the prefixes are written (3). The next
  // terminal's barrier (1) also ends this one's reads of the prefixes, the
  // layout and this row buffer.
  int step = 0;
  for (int ti = t0; ti < t1;) {
    const int buf = step & 1;
    step++;
    const bool first = DYN && ti == cbeg;
    if (first && tid == 0) s_claim[1] = (int)atomicAdd(counter, (uint32_t)FAST_DYN_CHUNK);
    const R* r = rbuf + (size_t)buf * A.stride;
    // Row ti landed (own copies), partial maxima published.
    cp_async_wait_all();
    R mx = 0;
    if constexpr (F64) {
      for (int i = tid; i < hpo / 2; i += FAST_THREADS) {
        const double2 v = reinterpret_cast<const double2*>(r)[i];
        mx = row_max(mx, row_max(v.x, v.y));
      }
    } else {
      for (int i = tid; i < hpo / 4; i += FAST_THREADS) {
        const float4 v = reinterpret_cast<const float4*>(r)[i];
        mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) mx = row_max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    if (lane == 0) fred[buf * (FAST_THREADS / 32) + warp] = mx;
    __syncthreads();  // (1)
    // The task after ti: the next in its range, or (DYN) the first of the
    // chunk claimed while this chunk started.
    int next;
    if constexpr (DYN) {
      if (first) claimed = s_claim[1];
      next = ti + 1 < cend ? ti + 1 : min(claimed, t1);
    } else {
      next = ti + 1;
    }
    if (next < t1) prefetch(next, buf ^ 1);
    const FastTask cur = T;
    if (next < t1) T = tasks[next];  // next task's record, loaded early
    if (DYN && next != ti + 1) {
      cbeg = next;
      cend = min(t1, next + FAST_DYN_CHUNK);
    }
    ti = next;
    if (A.alive[cur.slot] == 0) continue;  // dead subtree (cfr.rs:267-274): row untouched
    if (cur.board != board) {
      board = cur.board;
      const size_t lay = (size_t)board * 2 + p;
      const uint16_t* gseg = A.seg + lay * FAST_SEGS;
      if (tid < FAST_SEGS) sseg[tid] = gseg[tid];
      L = gseg[FAST_SEGS - 1];
      const uint16_t* gcat = A.cat + lay * A.cstride;
      for (int k = tid; k < L; k += FAST_THREADS) scat[k] = gcat[k];
      const uint4* grec = A.rec + lay * A.tstride;
      for (int h = tid; h < np; h += FAST_THREADS) srec[h] = grec[h];
      __syncthreads();  // the new layout is staged (once per board)
    }
    mx = 0;
#pragma unroll
    for (int w = 0; w < FAST_THREADS / 32; w++) mx = row_max(mx, fred[buf * (FAST_THREADS / 32) + w]);
    const int S = scale_exponent(mx);
    const double scale = pow2(S), inv = pow2(-S);
    const double pa = cur.a * inv, pb = cur.b * inv, pc = cur.c * inv, pd = cur.d * inv;

    // This thread's E consecutive layout elements, straight from the row.
    constexpr int N = FAST_THREADS * E;
    long long x[E];
    long long local = 0;
#pragma unroll
    for (int i = 0; i < E; i++) {
      const int k = tid * E + i;
      x[i] = k < L ? fixed(r[scat[k]], scale) : 0ll;
      local += x[i];
    }
    long long inc = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();  // (2)
    long long acc = inc - local;
#pragma unroll
    for (int w = 0; w < FAST_THREADS / 32; w++)
      if (w < warp) acc += wsum[w];
    long long* own = G + tid * E;
#pragma unroll
    for (int i = 0; i < E; i++) {
      own[i] = acc;
      acc += x[i];
    }
    if (tid == FAST_THREADS - 1) G[N] = acc;
    __syncthreads();  // (3)

    // Values in hand order. Card c's segment runs from sseg[1+c] to sseg[2+c].
    const long long T0 = G[sseg[1]];
    R* out = A.vals + (size_t)cur.row * A.stride;
    R* fout = cur.frow != NONE32 ? A.vals + (size_t)cur.frow * A.stride : nullptr;
    const uint32_t kind = cur.kind;
    const bool fold = kind == T_FOLD_SCALAR || kind == T_FOLD_BATCH;
    const bool scalar = kind == T_FOLD_SCALAR || kind == T_SHOWDOWN_SCALAR;
#pragma unroll 2
    for (int h = tid; h < hpp; h += FAST_THREADS) {
      R v = 0, fv = 0;
      if (h < np) {
        const uint4 q = srec[h];
        const int a = (int)(q.w & 0xFF), b = (int)((q.w >> 8) & 0xFF);
        const long long a0 = G[sseg[1 + a]], b0 = G[sseg[1 + b]];
        const longlong2 ca = make_longlong2(a0, G[sseg[2 + a]] - a0);
        const longlong2 cb = make_longlong2(b0, G[sseg[2 + b]] - b0);
        const uint16_t sm = ssame[h];
        const long long si = sm == 0xFFFF ? 0ll : fixed(r[sm], scale);
        const long long F = T0 - ca.y - cb.y + si;
        if constexpr (F64) {
          // Double rows: every value in double, no f32 rounding.
          if (fold) {
            v = pa * (double)F;
          } else {
            if (q.w >> 16) {
              const long long Gw = G[q.x & 0xFFFF], Gs = G[q.x >> 16];
              const long long Gaw = G[q.y & 0xFFFF], Gas = G[q.y >> 16];
              const long long Gbw = G[q.z & 0xFFFF], Gbs = G[q.z >> 16];
              const long long W = (Gw + ca.x + cb.x) - Gaw - Gbw;
              const long long Lx = (T0 + Gas + Gbs) - Gs - (ca.x + ca.y) - (cb.x + cb.y);
              double res = pa * (double)W + pb * (double)Lx;
              if (pc != 0.0) {
                const long long eq = (Gs - Gw) - (Gas - Gaw) - (Gbs - Gbw) + si;
                res += pc * (double)eq;
              }
              v = res;
            }
            if (fout) fv = pd * (double)F;
          }
        } else if (fold) {
          // eval_fold (eval.rs:40-64) returns zeros on a zero total.
          v = (scalar && T0 == 0) ? 0.0f : (float)(pa * (double)F);
        } else {
          if (q.w >> 16) {
            const long long Gw = G[q.x & 0xFFFF], Gs = G[q.x >> 16];
            const long long Gaw = G[q.y & 0xFFFF], Gas = G[q.y >> 16];
            const long long Gbw = G[q.z & 0xFFFF], Gbs = G[q.z >> 16];
            // weaker: Gw - (Gaw - C0a) - (Gbw - C0b); stronger: (T0 - Gs)
            // - (CTa - (Gas - C0a)) - (CTb - (Gbs - C0b)).
            const long long W = (Gw + ca.x + cb.x) - Gaw - Gbw;
            const long long Lx = (T0 + Gas + Gbs) - Gs - (ca.x + ca.y) - (cb.x + cb.y);
            if (scalar) {
              v = (float)(pa * (double)W) + (float)(pb * (double)Lx);
            } else {
              double res = pa * (double)W;
              res += pb * (double)Lx;
              v = (float)res;
            }
            if (cur.c != 0.0) {
              const long long eq = (Gs - Gw) - (Gas - Gaw) - (Gbs - Gbw) + si;
              v += (float)(pc * (double)eq);
            }
          }
          if (fout) fv = (float)(pd * (double)F);
        }
      }
      out[h] = v;
      if (fout) fout[h] = fv;
    }
  }
  cp_async_wait_all();
}

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum less the kernel's own static shared memory (the two together may
// not pass the opt-in maximum).
static cudaError_t allow_dynamic_smem(const void* fn, int optin) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

template <int E>
static cudaError_t setup_e(int optin, size_t smem, int& blocks) {
  cudaError_t e = allow_dynamic_smem((const void*)fast_terminal_kernel<E, float>, optin);
  if (e != cudaSuccess) return e;
  e = allow_dynamic_smem((const void*)fast_terminal_kernel<E, double>, optin);
  if (e != cudaSuccess) return e;
  e = allow_dynamic_smem((const void*)fast_terminal_kernel<E, float, true>, optin);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fast_terminal_kernel<E, float>, FAST_THREADS, smem);
}

int fast_emax(int tstride) {
  const int e = (3 * tstride + FAST_THREADS - 1) / FAST_THREADS;
  return e | 1;  // odd: conflict-free strided 8-byte access
}

size_t fast_smem_bytes(int stride, int emax, int cstride, int tstride, int rsize) {
  return FastSmem(stride, emax, cstride, tstride, rsize).total;
}

int fast_blocks_per_sm(int stride, int emax, int cstride, int tstride) {
  int blocks = 0;
  const size_t smem = fast_smem_bytes(stride, emax, cstride, tstride, 4);
  // The limit is the device's opt-in maximum (a per-kernel setting shared by
  // every handle), not this handle's size.
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  if ((size_t)optin < fast_smem_bytes(stride, emax, cstride, tstride, 8)) return 0;
  cudaError_t e = cudaErrorInvalidValue;
  switch (emax) {
#define FAST_E(e_)                          \
  case e_:                                  \
    e = setup_e<e_>(optin, smem, blocks);   \
    break;
    FAST_E(1) FAST_E(3) FAST_E(5) FAST_E(7) FAST_E(9) FAST_E(11) FAST_E(13) FAST_E(15) FAST_E(17)
#undef FAST_E
  }
  return e == cudaSuccess ? blocks : 0;
}

// ---------------------------------------------------------------------------
// Warp-per-terminal evaluation: the solve's terminal kernel.
//
// The same fixed-point prefix sums as fast_terminal_kernel, but every
// terminal is evaluated by one warp with no block barrier inside a task.
// Block b takes the contiguous task range [b N / G, (b+1) N / G) of the N
// tasks (ordered by layout); its warps take the range's tasks in turn
// (warp w: tasks w, w + W, ...). A unit is a maximal run of tasks on one
// layout; the block stages a unit's layout in shared memory once, with a
// block barrier only where its range crosses from one unit to the next.
// Per task and warp:
//   1. the reach row is copied to the warp's shared row (16-byte loads) and
//      its maximum reduced across the warp, which fixes the scale 2^S;
//   2. each lane converts E consecutive layout elements to fixed point,
//      writes them and sums them; a warp shuffle scan turns the lane sums
//      into exclusive offsets and a second pass rewrites the elements as
//      exclusive prefixes G;
//   3. each lane forms the values of hands lane, lane+32, ... from six
//      prefixes and the four card-segment bounds, exactly as
//      fast_terminal_kernel does, and stores them coalesced.
// Shared memory per block: the layout (elements, per-hand records,
// identical-hand map, segment starts) and, per warp, two rows (the current
// task's and the next one's, copied asynchronously) and the prefix array;
// the warp count W is a launch parameter.
struct WarpSmem {
  size_t same, cat, rec, seg, warp0, warp_bytes, row_bytes, total;
  __host__ __device__ WarpSmem(int stride, int cstride, int tstride, int rsize, int warps) {
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    same = 0;
    cat = up16(same + (size_t)stride * 2);
    rec = up16(cat + (size_t)cstride * 2);
    seg = up16(rec + (size_t)tstride * 16);
    warp0 = up16(seg + FAST_SEGS * 2);
    row_bytes = up16((size_t)stride * rsize);
    warp_bytes = 2 * row_bytes + up16(warp_prefix_entries(cstride) * 8);
    total = warp0 + (size_t)warps * warp_bytes;
  }
};

template <typename R>
__global__ void __launch_bounds__(512, 1) warp_terminal_kernel(FastArgsT<R> A, const FastTask* __restrict__ tasks,
                                                            const TermUnit* __restrict__ units, int nunits,
                                                            int ntasks) {
  extern __shared__ __align__(16) unsigned char smem_w[];
  const int W = (int)blockDim.x >> 5;
  const WarpSmem L_(A.stride, A.cstride, A.tstride, (int)sizeof(R), W);
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_w + L_.same);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_w + L_.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_w + L_.rec);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_w + L_.seg);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  R* row = reinterpret_cast<R*>(smem_w + L_.warp0 + (size_t)warp * L_.warp_bytes);
  long long* G = reinterpret_cast<long long*>(smem_w + L_.warp0 + (size_t)warp * L_.warp_bytes + 2 * L_.row_bytes);

  const int p = A.p;
  const int hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  for (int h = tid; h < hpp; h += blockDim.x) {
    const uint32_t sm = h < np ? A.same[h] : NONE32;
    ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
  }

  const int t0 = (int)(((long long)blockIdx.x * ntasks) / gridDim.x);
  const int t1 = (int)(((long long)(blockIdx.x + 1) * ntasks) / gridDim.x);
  // The unit holding task t0: units tile [0, ntasks) in order.
  int u = 0;
  {
    int hi = nunits - 1;
    while (u < hi) {
      const int mid = (u + hi) >> 1;
      if ((int)(units[mid].first + units[mid].count) <= t0) u = mid + 1;
      else hi = mid;
    }
  }
  // Each warp double-buffers reach rows: the row of its next task is copied
  // (cp.async) while the current task runs.
  R* const row_b = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(row) + L_.row_bytes);
  int buf = 0;
  int next = t0 + warp;  // this warp's current task
  bool live = false;
  if (next < t1) {
    live = A.alive[tasks[next].slot] != 0;
    if (live) warp_row_prefetch<R>(A, tasks[next].slot, row, lane);
  }
  cp_async_commit();
  for (; u < nunits && (int)units[u].first < t1; u++) {
    const TermUnit U = units[u];
    __syncthreads();  // the previous unit's warps are done with the layout
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
    const int end = min(t1, (int)(U.first + U.count));
    for (; next < end; next += W) {
      // The following task's row (it may lie in a later unit: rows do not
      // depend on the layout).
      const int nx = next + W;
      bool nlive = false;
      if (nx < t1) {
        const uint32_t ns = tasks[nx].slot;
        nlive = A.alive[ns] != 0;
        if (nlive) warp_row_prefetch<R>(A, ns, buf ? row : row_b, lane);
      }
      cp_async_commit();
      cp_async_wait<1>();  // this task's row has landed
      __syncwarp();
      // Dead subtree (cfr.rs:267-274): row untouched.
      if (live) warp_terminal_task<R, true>(A, tasks[next], Y, buf ? row_b : row, G, lane);
      live = nlive;
      buf ^= 1;
    }
  }
}

// The warp-per-terminal evaluation with dynamic scheduling. The static
// kernel above gives every block an equal share of the task list; the work
// is not equal (dead subtrees, cfr.rs:267-274, are skipped, and they gather
// in some parts of the tree as strategies sharpen), so some blocks finish
// long before others. Here blocks claim chunks of TERM_DYN_CHUNK consecutive
// tasks from a global counter (zeroed before the launch), stage the layout of
// each run of the chunk that lies on one layout, and their warps claim the
// run's tasks one at a time from a shared counter, prefetching the claimed
// task's row (cp.async) while the current one is evaluated.
constexpr int TERM_DYN_CHUNK = 128;
size_t warp_terminal_smem(int stride, int cstride, int tstride, int rsize, int warps);

template <typename R>
__global__ void __launch_bounds__(512, 1) warp_terminal_dyn_kernel(FastArgsT<R> A, const FastTask* __restrict__ tasks,
                                                                const TermUnit* __restrict__ units, int nunits,
                                                                int ntasks, uint32_t* __restrict__ counter) {
  extern __shared__ __align__(16) unsigned char smem_w[];
  const int W = (int)blockDim.x >> 5;
  const WarpSmem L_(A.stride, A.cstride, A.tstride, (int)sizeof(R), W);
  // The chunk's first task and the run's claim counter, after the warps' areas.
  int& s_base = reinterpret_cast<int*>(smem_w + L_.total)[0];
  int& s_next = reinterpret_cast<int*>(smem_w + L_.total)[1];
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_w + L_.same);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_w + L_.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_w + L_.rec);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_w + L_.seg);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  R* const row_a = reinterpret_cast<R*>(smem_w + L_.warp0 + (size_t)warp * L_.warp_bytes);
  R* const row_b = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(row_a) + L_.row_bytes);
  long long* G = reinterpret_cast<long long*>(smem_w + L_.warp0 + (size_t)warp * L_.warp_bytes + 2 * L_.row_bytes);

  const int p = A.p;
  const int hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  for (int h = tid; h < hpp; h += blockDim.x) {
    const uint32_t sm = h < np ? A.same[h] : NONE32;
    ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
  }
  uint32_t staged = NONE32;
  int L = 0;
  for (;;) {
    __syncthreads();  // the previous run is finished with the layout and the claim counter
    if (tid == 0) s_base = (int)atomicAdd(counter, (uint32_t)TERM_DYN_CHUNK);
    __syncthreads();
    const int base = s_base;
    if (base >= ntasks) break;
    const int end = min(ntasks, base + TERM_DYN_CHUNK);
    // The unit (maximal run on one layout) holding `base`.
    int u = 0;
    {
      int hi = nunits - 1;
      while (u < hi) {
        const int mid = (u + hi) >> 1;
        if ((int)(units[mid].first + units[mid].count) <= base) u = mid + 1;
        else hi = mid;
      }
    }
    for (int r0 = base; r0 < end; u++) {
      const TermUnit U = units[u];
      const int r1 = min(end, (int)(U.first + U.count));
      if (U.layout != staged) {  // block-uniform
        __syncthreads();  // the previous run's warps are done with the layout
        staged = U.layout;
        const size_t lay = (size_t)U.layout * 2 + p;
        const uint16_t* gseg = A.seg + lay * FAST_SEGS;
        if (tid < FAST_SEGS) sseg[tid] = gseg[tid];
        L = gseg[FAST_SEGS - 1];
        const uint16_t* gcat = A.cat + lay * A.cstride;
        for (int k = tid; k < L; k += blockDim.x) scat[k] = gcat[k];
        const uint4* grec = A.rec + lay * A.tstride;
        for (int h = tid; h < np; h += blockDim.x) srec[h] = grec[h];
      }
      if (tid == 0) s_next = r0;
      __syncthreads();  // the layout is staged and the claim counter set
      const WarpLayout Y{ssame, scat, srec, sseg, L};
      auto claim = [&]() {
        int t = 0;
        if (lane == 0) t = atomicAdd(&s_next, 1);
        return __shfl_sync(0xffffffffu, t, 0);
      };
      int cur = claim();
      bool live = cur < r1 && A.alive[tasks[cur].slot] != 0;
      if (live) warp_row_prefetch<R>(A, tasks[cur].slot, row_a, lane);
      cp_async_commit();
      int buf = 0;
      while (cur < r1) {
        const int nxt = claim();
        const bool nlive = nxt < r1 && A.alive[tasks[nxt].slot] != 0;
        if (nlive) warp_row_prefetch<R>(A, tasks[nxt].slot, buf ? row_a : row_b, lane);
        cp_async_commit();
        cp_async_wait<1>();  // this task's row has landed
        __syncwarp();
        // Dead subtree (cfr.rs:267-274): row untouched.
        if (live) warp_terminal_task<R, true>(A, tasks[cur], Y, buf ? row_b : row_a, G, lane);
        cur = nxt;
        live = nlive;
        buf ^= 1;
      }
      cp_async_wait<0>();
      __syncwarp();
      r0 = r1;
      __syncthreads();  // every warp has left this run's claim loop
    }
  }
}

void launch_warp_terminal_dyn(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                              int warps, int max_blocks, uint32_t* counter, cudaStream_t s) {
  if (nunits <= 0 || ntasks <= 0) return;
  const int chunks = (ntasks + TERM_DYN_CHUNK - 1) / TERM_DYN_CHUNK;
  const int blocks = chunks < max_blocks ? chunks : max_blocks;
  const size_t smem = warp_terminal_smem(A.stride, A.cstride, A.tstride, 4, warps) + 16;
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  warp_terminal_dyn_kernel<float><<<blocks, warps * 32, smem, s>>>(A, tasks, units, nunits, ntasks, counter);
}

// Warp count (1..max_warps) of the dynamically scheduled kernel that
// maximises resident warps per SM (its shared memory is the static kernel's
// plus 16 bytes of counters), and the blocks per SM at that count; 0 if none
// fits.
int warp_terminal_dyn_setup(int stride, int cstride, int tstride, int max_warps, int& blocks_per_sm) {
  int dev = 0, optin = 0;
  blocks_per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  const void* fn = (const void*)warp_terminal_dyn_kernel<float>;
  if (allow_dynamic_smem(fn, optin) != cudaSuccess) return 0;
  int best_w = 0, best_b = 0;
  for (int w = 1; w <= max_warps; w++) {
    const size_t smem = warp_terminal_smem(stride, cstride, tstride, 4, w) + 16;
    if (smem > (size_t)optin) break;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, w * 32, smem) != cudaSuccess) return 0;
    if (b > 0 && w * b >= best_w * best_b) {
      best_w = w;
      best_b = b;
    }
  }
  blocks_per_sm = best_b;
  return best_w;
}

size_t warp_terminal_smem(int stride, int cstride, int tstride, int rsize, int warps) {
  return WarpSmem(stride, cstride, tstride, rsize, warps).total;
}

// Warp count (1..max_warps) that maximises resident warps per SM for rows
// of rsize bytes, and the blocks per SM at that count; 0 if none fits.
int warp_terminal_setup(int stride, int cstride, int tstride, int rsize, int max_warps, int& blocks_per_sm) {
  int dev = 0, optin = 0;
  blocks_per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  const void* fn = rsize == 8 ? (const void*)warp_terminal_kernel<double> : (const void*)warp_terminal_kernel<float>;
  if (allow_dynamic_smem(fn, optin) != cudaSuccess) return 0;
  int best_w = 0, best_b = 0;
  for (int w = 1; w <= max_warps; w++) {
    const size_t smem = warp_terminal_smem(stride, cstride, tstride, rsize, w);
    if (smem > (size_t)optin) break;
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, w * 32, smem) != cudaSuccess) return 0;
    if (b > 0 && w * b >= best_w * best_b) {
      best_w = w;
      best_b = b;
    }
  }
  blocks_per_sm = best_b;
  return best_w;
}

template <typename R>
static void launch_warp_terminal_t(const FastArgsT<R>& A, const FastTask* tasks, const TermUnit* units, int nunits,
                                   int ntasks, int warps, int max_blocks, cudaStream_t s) {
  if (nunits <= 0 || ntasks <= 0) return;
  // At most one block per task: every block's range is non-empty.
  const int blocks = ntasks < max_blocks ? ntasks : max_blocks;
  const size_t smem = warp_terminal_smem(A.stride, A.cstride, A.tstride, (int)sizeof(R), warps);
  warp_terminal_kernel<R><<<blocks, warps * 32, smem, s>>>(A, tasks, units, nunits, ntasks);
}

void launch_warp_terminal(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                          int warps, int max_blocks, cudaStream_t s) {
  launch_warp_terminal_t(A, tasks, units, nunits, ntasks, warps, max_blocks, s);
}

void launch_warp_terminal64(const FastArgs64& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                            int warps, int max_blocks, cudaStream_t s) {
  launch_warp_terminal_t(A, tasks, units, nunits, ntasks, warps, max_blocks, s);
}

void launch_fast_layouts(const EntryD* tables, const uint32_t* count, int tstride, int nboards, const uint8_t* hc1_0,
                         const uint8_t* hc2_0, const uint8_t* hc1_1, const uint8_t* hc2_1, int n0, int n1,
                         uint16_t* cat, uint16_t* seg, uint4* rec, int cstride, cudaStream_t s) {
  const int n = (nboards + 1) * 2;
  fast_layout_kernel<<<(n + 63) / 64, 64, 0, s>>>(tables, count, tstride, nboards, hc1_0, hc2_0, hc1_1, hc2_1, n0, n1,
                                                  cat, seg, rec, cstride);
}

template <typename R>
static void launch_fast_terminal_t(const FastArgsT<R>& A, const FastTask* tasks, int ntasks, int max_blocks,
                                   cudaStream_t s) {
  if (ntasks <= 0) return;
  const int blocks = ntasks < max_blocks ? ntasks : max_blocks;
  const size_t smem = fast_smem_bytes(A.stride, A.emax, A.cstride, A.tstride, (int)sizeof(R));
  switch (A.emax) {
#define FAST_E(e_)                                                                     \
  case e_:                                                                             \
    fast_terminal_kernel<e_, R><<<blocks, FAST_THREADS, smem, s>>>(A, tasks, ntasks); \
    break;
    FAST_E(1) FAST_E(3) FAST_E(5) FAST_E(7) FAST_E(9) FAST_E(11) FAST_E(13) FAST_E(15) FAST_E(17)
#undef FAST_E
  }
}

void launch_fast_terminal_dyn(const FastArgs& A, const FastTask* tasks, int ntasks, int max_blocks, uint32_t* counter,
                              cudaStream_t s) {
  if (ntasks <= 0) return;
  const int chunks = (ntasks + FAST_DYN_CHUNK - 1) / FAST_DYN_CHUNK;
  const int blocks = chunks < max_blocks ? chunks : max_blocks;
  const size_t smem = fast_smem_bytes(A.stride, A.emax, A.cstride, A.tstride, 4);
  cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  switch (A.emax) {
#define FAST_E(e_)                                                                                        \
  case e_:                                                                                                \
    fast_terminal_kernel<e_, float, true><<<blocks, FAST_THREADS, smem, s>>>(A, tasks, ntasks, counter); \
    break;
    FAST_E(1) FAST_E(3) FAST_E(5) FAST_E(7) FAST_E(9) FAST_E(11) FAST_E(13) FAST_E(15) FAST_E(17)
#undef FAST_E
  }
}

void launch_fast_terminal(const FastArgs& A, const FastTask* tasks, int ntasks, int max_blocks, cudaStream_t s) {
  launch_fast_terminal_t(A, tasks, ntasks, max_blocks, s);
}

void launch_fast_terminal64(const FastArgs64& A, const FastTask* tasks, int ntasks, int max_blocks, cudaStream_t s) {
  launch_fast_terminal_t(A, tasks, ntasks, max_blocks, s);
}

}  // namespace dcfr
