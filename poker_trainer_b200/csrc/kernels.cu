// sm_100a kernels of libdcfr.
//
// Every f32/f64 operation of the solve is performed in the order of the
// reference CPU solver (AhanDatta/Poker-Trainer crates/solver/src/cfr.rs,
// river.rs, eval.rs) and the library is compiled with -fmad=false, IEEE
// division and denormals kept, so results are bit-identical to it:
//   * row kernels (down_kernel / up_kernel) work on 4 hands per thread with
//     128-bit loads and stores; all their arithmetic is per hand;
//   * chance sums accumulate children in f64 in card order, then the
//     isomorphic cards through the suit permutation (cfr.rs:462-478);
//   * terminal values are in terminal.cu.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "row_items.cuh"

namespace dcfr {

// ------------------------------------------------------------ level kernels
// One launch per level, one block per node. Levels are chained with programmatic dependent
// launch: a level's grid is launched while the previous one drains and waits
// (griddepcontrol.wait) until that grid has completed and its writes are
// visible.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// COMP: 16-bit compressed storage (one block covers a node's row).
template <int MODE, int MAXA, bool COMP>
__global__ void __launch_bounds__(ROW_MAX_THREADS) down_kernel(RowArgs A, const DownTask* __restrict__ tasks,
                                                               int chunks) {
  const int t = blockIdx.x / chunks, ch = blockIdx.x - t * chunks;
  const DownTask T = tasks[t];  // plan data: readable before the wait
  pdl_wait();
  const int h0 = (ch * (int)blockDim.x + (int)threadIdx.x) * VEC;
  int phase = 0;  // block_max scratch row (compressed storage)
  if (T.kind == D_OPP_SPLIT) down_item<MODE, MAXA, D_OPP_SPLIT, COMP>(A, T, h0, threadIdx.x & 31, &phase);
  else down_item<MODE, 1, D_CHANCE_SPLIT>(A, T, h0, threadIdx.x & 31);
  pdl_launch_dependents();
}

template <int MODE, int MAXA, bool COMP>
__global__ void __launch_bounds__(ROW_MAX_THREADS) up_kernel(RowArgs A, const UpTask* __restrict__ tasks, int chunks) {
  const int t = blockIdx.x / chunks, ch = blockIdx.x - t * chunks;
  const UpTask T = tasks[t];
  pdl_wait();
  const int h0 = (ch * (int)blockDim.x + (int)threadIdx.x) * VEC;
  int phase = 0;  // block_max scratch row (compressed storage)
  if (T.kind == U_OWN) up_item<MODE, MAXA, U_OWN, COMP>(A, T, h0, &phase);
  else if (T.kind == U_OPP_SUM) up_item<MODE, MAXA, U_OPP_SUM>(A, T, h0);
  else up_item<MODE, 1, U_CHANCE_SUM>(A, T, h0);
  pdl_launch_dependents();
}

// Fused river subtrees: one block per subtree walks its nodes (see
// FusedTree). Every thread keeps the same 4 hands throughout, so a node's
// rows are produced and consumed by the same threads; the barrier between
// down levels publishes the children's liveness flags.
template <int MODE, int MAXA, bool COMP>
__global__ void __launch_bounds__(ROW_MAX_THREADS) fused_down_kernel(RowArgs A, const FusedTree* __restrict__ trees,
                                                                     const DownTask* __restrict__ tasks) {
  const FusedTree F = trees[blockIdx.x];
  pdl_wait();
  const int h0 = (int)threadIdx.x * VEC, lane = threadIdx.x & 31;
  int phase = 0;  // block_max scratch row (compressed storage)
#pragma unroll 1
  for (uint32_t i = 0; i < F.down_count; i++) {
    const DownTask T = tasks[F.down_first + i];
    if (T.kind & LEVEL_BREAK) __syncthreads();
    down_item<MODE, MAXA, D_OPP_SPLIT, COMP>(A, T, h0, lane, &phase);
  }
  pdl_launch_dependents();
}

template <int MODE, int MAXA, bool COMP>
__global__ void __launch_bounds__(ROW_MAX_THREADS) fused_up_kernel(RowArgs A, const FusedTree* __restrict__ trees,
                                                                   const UpTask* __restrict__ tasks) {
  const FusedTree F = trees[blockIdx.x];
  pdl_wait();
  const int h0 = (int)threadIdx.x * VEC;
  int phase = 0;  // block_max scratch row (compressed storage)
#pragma unroll 1
  for (uint32_t i = 0; i < F.up_count; i++) {
    const UpTask T = tasks[F.up_first + i];
    if ((T.kind & KIND_MASK) == U_OWN) up_item<MODE, MAXA, U_OWN, COMP>(A, T, h0, &phase);
    else up_item<MODE, MAXA, U_OPP_SUM>(A, T, h0);
  }
  pdl_launch_dependents();
}

// ------------------------------------------------------------ setup kernels
// 7-card strength (crates/holdem/src/eval.rs:104-198): category<<26 | payload.
__device__ __forceinline__ uint32_t hb(uint32_t x) { return 31u - (uint32_t)__clz(x); }

__device__ uint32_t topb(uint32_t x, uint32_t n) {
  uint32_t out = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (x == 0) break;
    uint32_t b = 1u << hb(x);
    out |= b;
    x ^= b;
  }
  return out;
}

__device__ int straight_top(uint32_t ranks) {
  uint32_t run = ranks & (ranks << 1) & (ranks << 2) & (ranks << 3) & (ranks << 4);
  if (run) return (int)hb(run);
  if ((ranks & 0x100Fu) == 0x100Fu) return 3;
  return -1;
}

__device__ uint32_t strength_of(uint64_t mask) {
  uint32_t s[4] = {(uint32_t)(mask & 0x1FFF), (uint32_t)((mask >> 16) & 0x1FFF), (uint32_t)((mask >> 32) & 0x1FFF),
                   (uint32_t)((mask >> 48) & 0x1FFF)};
  for (int k = 0; k < 4; k++)
    if (__popc(s[k]) >= 5) {
      int h = straight_top(s[k]);
      return h >= 0 ? (8u << 26) | (uint32_t)h : (5u << 26) | topb(s[k], 5);
    }
  uint32_t any = s[0] | s[1] | s[2] | s[3];
  uint32_t two = (s[0] & s[1]) | (s[0] & s[2]) | (s[0] & s[3]) | (s[1] & s[2]) | (s[1] & s[3]) | (s[2] & s[3]);
  uint32_t three = (s[0] & s[1] & s[2]) | (s[0] & s[1] & s[3]) | (s[0] & s[2] & s[3]) | (s[1] & s[2] & s[3]);
  uint32_t four = s[0] & s[1] & s[2] & s[3];
  if (four) {
    uint32_t q = hb(four);
    return (7u << 26) | (q << 13) | topb(any & ~(1u << q), 1);
  }
  if (three) {
    uint32_t t = hb(three);
    uint32_t rest = two & ~(1u << t);
    if (rest) return (6u << 26) | (t << 13) | (1u << hb(rest));
  }
  int h = straight_top(any);
  if (h >= 0) return (4u << 26) | (uint32_t)h;
  if (three) {
    uint32_t t = hb(three);
    return (3u << 26) | (t << 13) | topb(any & ~(1u << t), 2);
  }
  if (__popc(two) >= 2) {
    uint32_t pairs = topb(two, 2);
    return (2u << 26) | (pairs << 13) | topb(any & ~pairs, 1);
  }
  if (two) {
    uint32_t pp = hb(two);
    return (1u << 26) | (pp << 13) | topb(any & ~(1u << pp), 3);
  }
  return topb(any, 5);
}

__device__ __forceinline__ uint64_t lane_bit(int c) { return 1ull << ((c & 3) * 16 + (c >> 2)); }

// One block per (board, player): strengths of the player's hands that don't
// touch the board, sorted by (strength, hand index) — StrengthTable::new
// (crates/solver/src/hands.rs:137-158).
constexpr int SORT_N = 2048;
__global__ void __launch_bounds__(512) strength_kernel(const uint8_t* __restrict__ boards, const uint8_t* hc1_0,
                                                       const uint8_t* hc2_0, const uint8_t* hc1_1,
                                                       const uint8_t* hc2_1, int n0, int n1, EntryD* out,
                                                       uint32_t* count, int tstride) {
  __shared__ unsigned long long keys[SORT_N];
  const int b = blockIdx.x >> 1, q = blockIdx.x & 1;
  const uint8_t* c1 = q ? hc1_1 : hc1_0;
  const uint8_t* c2 = q ? hc2_1 : hc2_0;
  const int n = q ? n1 : n0;
  uint64_t mask = 0, set = 0;
  for (int k = 0; k < 5; k++) {
    int c = boards[b * 5 + k];
    mask |= lane_bit(c);
    set |= 1ull << c;
  }
  int valid_local = 0;
  for (int i = threadIdx.x; i < SORT_N; i += blockDim.x) {
    unsigned long long key = ~0ull;
    if (i < n) {
      int a = c1[i], bb = c2[i];
      if (!((set >> a) & 1) && !((set >> bb) & 1)) {
        uint32_t st = strength_of(mask | lane_bit(a) | lane_bit(bb));
        key = ((unsigned long long)st << 32) | ((unsigned long long)i << 16) | ((unsigned long long)a << 8) |
              (unsigned long long)bb;
        valid_local++;
      }
    }
    keys[i] = key;
  }
  __syncthreads();
  // Bitonic sort, ascending.
  for (int k = 2; k <= SORT_N; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int i = threadIdx.x; i < SORT_N; i += blockDim.x) {
        int ixj = i ^ jj;
        if (ixj > i) {
          unsigned long long x = keys[i], y = keys[ixj];
          bool up = (i & k) == 0;
          if ((x > y) == up) {
            keys[i] = y;
            keys[ixj] = x;
          }
        }
      }
      __syncthreads();
    }
  }
  __shared__ int total;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  atomicAdd(&total, valid_local);
  __syncthreads();
  const int cnt = total;
  EntryD* dst = out + (size_t)blockIdx.x * tstride;
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) {
    unsigned long long k = keys[i];
    EntryD e;
    e.strength = (uint32_t)(k >> 32);
    e.idx = (uint16_t)((k >> 16) & 0xFFFF);
    e.c1 = (uint8_t)((k >> 8) & 0xFF);
    e.c2 = (uint8_t)(k & 0xFF);
    dst[i] = e;
  }
  if (threadIdx.x == 0) count[blockIdx.x] = (uint32_t)cnt;
}

// Strengths of explicit 5..7-card hands given as eval lane masks (tests of
// the device evaluator against the reference's).
__global__ void evaluate_kernel(const unsigned long long* masks, uint32_t* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = strength_of(masks[i]);
}

// All 2,598,960 five-card hands, per-category counts (eval.rs:246-265).
__global__ void five_card_counts_kernel(unsigned long long* counts) {
  __shared__ unsigned int local[9];
  if (threadIdx.x < 9) local[threadIdx.x] = 0;
  __syncthreads();
  // blockIdx.x enumerates (a, b) pairs; threads enumerate (c, d, e).
  int a = 0, b = 0, idx = blockIdx.x;
  for (a = 0; a < 52; a++) {
    int nb = 51 - a;
    if (idx < nb) {
      b = a + 1 + idx;
      break;
    }
    idx -= nb;
  }
  uint64_t m2 = lane_bit(a) | lane_bit(b);
  for (int t = threadIdx.x; t < 52 * 52; t += blockDim.x) {
    int c = t / 52, d = t % 52;
    if (c <= b || d <= c) continue;
    uint64_t m4 = m2 | lane_bit(c) | lane_bit(d);
    for (int e = d + 1; e < 52; e++) atomicAdd(&local[strength_of(m4 | lane_bit(e)) >> 26], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 9) atomicAdd(&counts[threadIdx.x], (unsigned long long)local[threadIdx.x]);
}

// ---------------------------------------------------------- host launchers
// One block per node (and chunk of 4 * ROW_MAX_THREADS hands): a thread per 4
// hands, whole warps. Launched with programmatic stream serialization so the
// grid is set up while the previous level drains; the kernel waits
// (griddepcontrol.wait) before touching rows or storage.
static int row_threads(int hp) {
  const int t = ((hp + VEC - 1) / VEC + 31) / 32 * 32;
  return t < 32 ? 32 : (t > ROW_MAX_THREADS ? ROW_MAX_THREADS : t);
}

template <typename K, typename Task>
static void launch_level(K kernel, const RowArgs& A, const Task* tasks, int ntasks, int hp, cudaStream_t s) {
  const int threads = row_threads(hp), chunks = (hp + threads * VEC - 1) / (threads * VEC);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ntasks * chunks));
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, A, tasks, chunks);
}

template <int MODE>
static void launch_down_m(int maxa, const RowArgs& A, const DownTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (A.compressed) {
    if (maxa <= 4) return launch_level(down_kernel<MODE, 4, true>, A, tasks, ntasks, hp, s);
    if (maxa <= 8) return launch_level(down_kernel<MODE, 8, true>, A, tasks, ntasks, hp, s);
    return launch_level(down_kernel<MODE, MAX_ACTIONS, true>, A, tasks, ntasks, hp, s);
  }
  if (maxa <= 4) return launch_level(down_kernel<MODE, 4, false>, A, tasks, ntasks, hp, s);
  if (maxa <= 8) return launch_level(down_kernel<MODE, 8, false>, A, tasks, ntasks, hp, s);
  launch_level(down_kernel<MODE, MAX_ACTIONS, false>, A, tasks, ntasks, hp, s);
}

template <int MODE>
static void launch_up_m(int maxa, const RowArgs& A, const UpTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (A.compressed) {
    if (maxa <= 4) return launch_level(up_kernel<MODE, 4, true>, A, tasks, ntasks, hp, s);
    if (maxa <= 8) return launch_level(up_kernel<MODE, 8, true>, A, tasks, ntasks, hp, s);
    return launch_level(up_kernel<MODE, MAX_ACTIONS, true>, A, tasks, ntasks, hp, s);
  }
  if (maxa <= 4) return launch_level(up_kernel<MODE, 4, false>, A, tasks, ntasks, hp, s);
  if (maxa <= 8) return launch_level(up_kernel<MODE, 8, false>, A, tasks, ntasks, hp, s);
  launch_level(up_kernel<MODE, MAX_ACTIONS, false>, A, tasks, ntasks, hp, s);
}

template <typename K, typename Task>
static void launch_fused(K kernel, const RowArgs& A, const FusedTree* trees, int ntrees, const Task* tasks, int hp,
                         cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ntrees);
  cfg.blockDim = dim3((unsigned)row_threads(hp));
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, A, trees, tasks);
}

template <int MODE>
static void launch_fused_m(bool up, int maxa, const RowArgs& A, const FusedTree* trees, int ntrees,
                           const DownTask* dt, const UpTask* ut, int hp, cudaStream_t s) {
  if (A.compressed) {
    if (up) {
      if (maxa <= 4) return launch_fused(fused_up_kernel<MODE, 4, true>, A, trees, ntrees, ut, hp, s);
      if (maxa <= 8) return launch_fused(fused_up_kernel<MODE, 8, true>, A, trees, ntrees, ut, hp, s);
      return launch_fused(fused_up_kernel<MODE, MAX_ACTIONS, true>, A, trees, ntrees, ut, hp, s);
    }
    if (maxa <= 4) return launch_fused(fused_down_kernel<MODE, 4, true>, A, trees, ntrees, dt, hp, s);
    if (maxa <= 8) return launch_fused(fused_down_kernel<MODE, 8, true>, A, trees, ntrees, dt, hp, s);
    return launch_fused(fused_down_kernel<MODE, MAX_ACTIONS, true>, A, trees, ntrees, dt, hp, s);
  }
  if (up) {
    if (maxa <= 4) return launch_fused(fused_up_kernel<MODE, 4, false>, A, trees, ntrees, ut, hp, s);
    if (maxa <= 8) return launch_fused(fused_up_kernel<MODE, 8, false>, A, trees, ntrees, ut, hp, s);
    return launch_fused(fused_up_kernel<MODE, MAX_ACTIONS, false>, A, trees, ntrees, ut, hp, s);
  }
  if (maxa <= 4) return launch_fused(fused_down_kernel<MODE, 4, false>, A, trees, ntrees, dt, hp, s);
  if (maxa <= 8) return launch_fused(fused_down_kernel<MODE, 8, false>, A, trees, ntrees, dt, hp, s);
  launch_fused(fused_down_kernel<MODE, MAX_ACTIONS, false>, A, trees, ntrees, dt, hp, s);
}

void launch_fused_down(int mode, int maxa, const RowArgs& A, const FusedTree* trees, int ntrees,
                       const DownTask* tasks, int hp, cudaStream_t s) {
  if (ntrees <= 0) return;
  if (mode == M_CFR) launch_fused_m<M_CFR>(false, maxa, A, trees, ntrees, tasks, nullptr, hp, s);
  else if (mode == M_BR) launch_fused_m<M_BR>(false, maxa, A, trees, ntrees, tasks, nullptr, hp, s);
  else launch_fused_m<M_AVG>(false, maxa, A, trees, ntrees, tasks, nullptr, hp, s);
}

void launch_fused_up(int mode, int maxa, const RowArgs& A, const FusedTree* trees, int ntrees, const UpTask* tasks,
                     int hp, cudaStream_t s) {
  if (ntrees <= 0) return;
  if (mode == M_CFR) launch_fused_m<M_CFR>(true, maxa, A, trees, ntrees, nullptr, tasks, hp, s);
  else if (mode == M_BR) launch_fused_m<M_BR>(true, maxa, A, trees, ntrees, nullptr, tasks, hp, s);
  else launch_fused_m<M_AVG>(true, maxa, A, trees, ntrees, nullptr, tasks, hp, s);
}

void launch_down(int mode, int maxa, const RowArgs& A, const DownTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (ntasks <= 0) return;
  if (mode == M_CFR) launch_down_m<M_CFR>(maxa, A, tasks, ntasks, hp, s);
  else if (mode == M_BR) launch_down_m<M_BR>(maxa, A, tasks, ntasks, hp, s);
  else launch_down_m<M_AVG>(maxa, A, tasks, ntasks, hp, s);
}

void launch_up(int mode, int maxa, const RowArgs& A, const UpTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (ntasks <= 0) return;
  if (mode == M_CFR) launch_up_m<M_CFR>(maxa, A, tasks, ntasks, hp, s);
  else if (mode == M_BR) launch_up_m<M_BR>(maxa, A, tasks, ntasks, hp, s);
  else launch_up_m<M_AVG>(maxa, A, tasks, ntasks, hp, s);
}

void launch_strength(const uint8_t* boards, int nboards, const uint8_t* hc1_0, const uint8_t* hc2_0,
                     const uint8_t* hc1_1, const uint8_t* hc2_1, int n0, int n1, EntryD* out, uint32_t* count,
                     int tstride, cudaStream_t s) {
  strength_kernel<<<nboards * 2, 512, 0, s>>>(boards, hc1_0, hc2_0, hc1_1, hc2_1, n0, n1, out, count, tstride);
}

void launch_evaluate(const unsigned long long* masks, uint32_t* out, int n, cudaStream_t s) {
  evaluate_kernel<<<(n + 255) / 256, 256, 0, s>>>(masks, out, n);
}

void launch_five_card_counts(unsigned long long* counts, cudaStream_t s) {
  five_card_counts_kernel<<<52 * 51 / 2, 256, 0, s>>>(counts);
}


// Start of a traversal: every liveness flag cleared but the root slot's, and
// the root's reach row copied into slot 0. One launch in place of two
// memsets and a copy, chained to the traversal's level launches by
// programmatic dependent launch (the flags are cleared only once the
// previous traversal's kernels, which read them, are complete). The first
// traversal of a DCFR iteration also advances the iteration (counter given):
// t += 1 and the iteration's discounts from the table, read by the
// traversal's row kernels after their wait.
__global__ void traversal_start_kernel(uint32_t* __restrict__ alive, int nslots, float* __restrict__ reach,
                                       const float* __restrict__ root_row, int stride, uint32_t* counter,
                                       const DiscountD* table, uint32_t table_len, DiscountD* cur) {
  pdl_wait();
  if (counter && blockIdx.x == 0 && threadIdx.x == 0) {
    const uint32_t t = *counter + 1;
    *counter = t;
    *cur = table[t < table_len ? t : table_len - 1];
  }
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x, step = gridDim.x * blockDim.x;
  for (int i = i0; i < nslots; i += step) alive[i] = i == 0 ? 1u : 0u;
  for (int i = i0; i < stride / 4; i += step)
    reinterpret_cast<float4*>(reach)[i] = reinterpret_cast<const float4*>(root_row)[i];
  pdl_launch_dependents();
}

// Storage blocks between the device layout (each action's row padded to hp
// entries) and the reference's packed layout (rows of n entries): a block of
// the grid per decision node, the elements copied as raw bits (f32 storage,
// or the 16-bit values of compressed storage). Unpacking zeroes the padding.
template <class T>
__global__ void __launch_bounds__(256) storage_pack_kernel(const T* __restrict__ dev, T* __restrict__ packed,
                                                            const StorageBlockD* __restrict__ blocks, int nblocks) {
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const StorageBlockD B = blocks[b];
    const uint32_t total = B.rows * B.n;
    for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
      const uint32_t a = i / B.n, h = i - a * B.n;
      packed[B.host + i] = dev[B.dev + (uint64_t)a * B.hp + h];
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) storage_unpack_kernel(T* __restrict__ dev, const T* __restrict__ packed,
                                                              const StorageBlockD* __restrict__ blocks, int nblocks) {
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const StorageBlockD B = blocks[b];
    const uint32_t total = B.rows * B.hp;
    for (uint32_t i = threadIdx.x; i < total; i += blockDim.x) {
      const uint32_t a = i / B.hp, h = i - a * B.hp;
      dev[B.dev + i] = h < B.n ? packed[B.host + (uint64_t)a * B.n + h] : T(0);
    }
  }
}

static int storage_grid(int nblocks) { return nblocks < 148 * 8 ? (nblocks > 0 ? nblocks : 1) : 148 * 8; }

void launch_storage_pack(int elem_bytes, const void* dev, void* packed, const StorageBlockD* blocks, int nblocks,
                         cudaStream_t s) {
  if (nblocks <= 0) return;
  if (elem_bytes == 4)
    storage_pack_kernel<uint32_t><<<storage_grid(nblocks), 256, 0, s>>>(
        static_cast<const uint32_t*>(dev), static_cast<uint32_t*>(packed), blocks, nblocks);
  else
    storage_pack_kernel<uint16_t><<<storage_grid(nblocks), 256, 0, s>>>(
        static_cast<const uint16_t*>(dev), static_cast<uint16_t*>(packed), blocks, nblocks);
}

void launch_storage_unpack(int elem_bytes, void* dev, const void* packed, const StorageBlockD* blocks, int nblocks,
                           cudaStream_t s) {
  if (nblocks <= 0) return;
  if (elem_bytes == 4)
    storage_unpack_kernel<uint32_t><<<storage_grid(nblocks), 256, 0, s>>>(
        static_cast<uint32_t*>(dev), static_cast<const uint32_t*>(packed), blocks, nblocks);
  else
    storage_unpack_kernel<uint16_t><<<storage_grid(nblocks), 256, 0, s>>>(
        static_cast<uint16_t*>(dev), static_cast<const uint16_t*>(packed), blocks, nblocks);
}

void launch_traversal_start(uint32_t* alive, int nslots, float* reach, const float* root_row, int stride,
                            uint32_t* counter, const DiscountD* table, uint32_t table_len, DiscountD* cur,
                            cudaStream_t s) {
  const int threads = 256, work = nslots > stride / 4 ? nslots : stride / 4;
  int blocks = (work + threads - 1) / threads;
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)blocks);
  cfg.blockDim = dim3((unsigned)threads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, traversal_start_kernel, alive, nslots, reach, root_row, stride, counter, table, table_len,
                     cur);
}

}  // namespace dcfr
