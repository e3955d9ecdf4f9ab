// FP64 best-response oracle on the GPU: the exploitability check of a solve
// (cfr::exploitability, crates/solver/src/cfr.rs:482-502) repeated with every
// reach and value row in double. This is the one step of the solve kept in
// FP64.
//
// It walks the same traversal plans as the f32 solve:
// - down: opponent nodes split the reach by the average strategy, computed in
//   double from the f32 strategy sums (normalize_in_place, cfr.rs:124-154);
//   chance nodes multiply by the chance factor and zero the opponent hands
//   that hold the dealt card;
// - terminals: fast_terminal_kernel<E, double> (terminal_fast.cu), with exact
//   fixed-point sums and double payoffs;
// - up: traverser nodes take the best action (best response) or the
//   average-strategy mix (raked games subtract the average EV); opponent and
//   chance nodes sum their children in double, chance children with the
//   traverser's blocked hands zeroed and isomorphic cards read through the
//   suit permutation (cfr.rs:462-478).
// The dead-subtree rule (cfr.rs:267-274) is kept: a slot whose reach row is
// all zero is skipped, and its parent never reads its rows.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"

namespace dcfr {

namespace {

constexpr int V64 = 4;  // hands per thread (two 16-byte loads of double2)

template <typename T>
__device__ __forceinline__ T pick64(int q, const T (&v)[2]) {
  return q ? v[1] : v[0];
}

__device__ __forceinline__ void ld4d(const double* p, double (&x)[V64]) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  x[0] = a.x;
  x[1] = a.y;
  x[2] = b.x;
  x[3] = b.y;
}
__device__ __forceinline__ void st4d(double* p, const double (&x)[V64]) {
  reinterpret_cast<double2*>(p)[0] = make_double2(x[0], x[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(x[2], x[3]);
}

// Opponent split by the average strategy, or chance split.
// One node's strategy sums for 4 hands as f32: stored f32, or the 16-bit
// sums decoded with the node's scale (load_strat, storage.rs:256-268).
__device__ __forceinline__ float4 sums4(const Row64Args& A, uint64_t store, uint32_t slot, size_t off) {
  if (A.sq == nullptr) return *reinterpret_cast<const float4*>(A.sums + store + off);
  const float sc = A.sscale[slot] / 65535.0f;
  const ushort4 q = *reinterpret_cast<const ushort4*>(A.sq + store + off);
  return make_float4((float)q.x * sc, (float)q.y * sc, (float)q.z * sc, (float)q.w * sc);
}

__device__ void down64_item(const Row64Args& A, const DownTask& T, int h0, int lane) {
  if (A.alive[T.in_slot] == 0) return;
  const int o = A.p ^ 1;
  const int hp = pick64(o, A.hp);
  const bool valid = h0 < hp;
  const size_t stride = (size_t)A.stride;
  double r[V64] = {0.0, 0.0, 0.0, 0.0};
  if (valid) ld4d(A.reach + (size_t)T.in_slot * stride + h0, r);
  if ((T.kind & KIND_MASK) == D_OPP_SPLIT) {
    const int na = (int)T.nchild;
    double tot[V64] = {0.0, 0.0, 0.0, 0.0};
    for (int a = 0; a < na; a++)
      if (valid) {
        const float4 s = sums4(A, T.store, T.cards, (size_t)a * hp + h0);
        tot[0] += (double)s.x;
        tot[1] += (double)s.y;
        tot[2] += (double)s.z;
        tot[3] += (double)s.w;
      }
    for (int a = 0; a < na; a++) {
      double c[V64] = {0.0, 0.0, 0.0, 0.0};
      if (valid) {
        const float4 s = sums4(A, T.store, T.cards, (size_t)a * hp + h0);
        const double sv[V64] = {(double)s.x, (double)s.y, (double)s.z, (double)s.w};
#pragma unroll
        for (int j = 0; j < V64; j++) {
          const double sigma = tot[j] > 0.0 ? sv[j] / tot[j] : 1.0 / (double)na;
          c[j] = sigma * r[j];
        }
        st4d(A.reach + (size_t)(T.out_slot + a) * stride + h0, c);
      }
      const bool nz = c[0] != 0.0 || c[1] != 0.0 || c[2] != 0.0 || c[3] != 0.0;
      if (__any_sync(0xffffffffu, valid && nz) && lane == 0) A.alive[T.out_slot + a] = 1u;
    }
  } else {
    uchar4 oc1 = make_uchar4(255, 255, 255, 255), oc2 = oc1;
    if (valid) {
      oc1 = *reinterpret_cast<const uchar4*>(pick64(o, A.hc1) + h0);
      oc2 = *reinterpret_cast<const uchar4*>(pick64(o, A.hc2) + h0);
    }
    const double factor = (double)T.factor;
    const uint8_t* cards = A.chance_cards + T.cards;
    for (uint32_t i = 0; i < T.nchild; i++) {
      const uint8_t card = cards[i];
      double c[V64];
#pragma unroll
      for (int j = 0; j < V64; j++) {
        const uint8_t a1 = (&oc1.x)[j], a2 = (&oc2.x)[j];
        c[j] = (a1 == card || a2 == card) ? 0.0 : r[j] * factor;
      }
      if (valid) st4d(A.reach + (size_t)(T.out_slot + i) * stride + h0, c);
      const bool nz = c[0] != 0.0 || c[1] != 0.0 || c[2] != 0.0 || c[3] != 0.0;
      if (__any_sync(0xffffffffu, valid && nz) && lane == 0) A.alive[T.out_slot + i] = 1u;
    }
  }
}

// Best response (MODE M_BR) or average-strategy value (M_AVG) of traverser
// nodes; sums of opponent and chance nodes.
template <int MODE>
__device__ void up64_item(const Row64Args& A, const UpTask& T, int h0) {
  if (A.alive[T.slot] == 0) return;
  const int p = A.p;
  const int hp = pick64(p, A.hp);
  if (h0 >= hp) return;
  const size_t stride = (size_t)A.stride;
  double out[V64] = {0.0, 0.0, 0.0, 0.0};
  const uint32_t kind = T.kind & KIND_MASK;
  if (kind == U_OWN) {
    const int na = (int)T.nchild;
    if (MODE == M_BR) {
      ld4d(A.vals + (size_t)T.child * stride + h0, out);
      for (int a = 1; a < na; a++) {
        double v[V64];
        ld4d(A.vals + (size_t)(T.child + a) * stride + h0, v);
#pragma unroll
        for (int j = 0; j < V64; j++) out[j] = v[j] > out[j] ? v[j] : out[j];
      }
    } else {
      double tot[V64] = {0.0, 0.0, 0.0, 0.0};
      for (int a = 0; a < na; a++) {
        const float4 s = sums4(A, T.store, T.cards, (size_t)a * hp + h0);
        tot[0] += (double)s.x;
        tot[1] += (double)s.y;
        tot[2] += (double)s.z;
        tot[3] += (double)s.w;
      }
      for (int a = 0; a < na; a++) {
        const float4 s = sums4(A, T.store, T.cards, (size_t)a * hp + h0);
        const double sv[V64] = {(double)s.x, (double)s.y, (double)s.z, (double)s.w};
        double v[V64];
        ld4d(A.vals + (size_t)(T.child + a) * stride + h0, v);
#pragma unroll
        for (int j = 0; j < V64; j++) out[j] += (tot[j] > 0.0 ? sv[j] / tot[j] : 1.0 / (double)na) * v[j];
      }
    }
  } else if (kind == U_OPP_SUM) {
    for (uint32_t a = 0; a < T.nchild; a++)
      if (A.alive[T.child_slot + a] != 0) {
        double v[V64];
        ld4d(A.vals + (size_t)(T.child + a) * stride + h0, v);
#pragma unroll
        for (int j = 0; j < V64; j++) out[j] += v[j];
      }
  } else {
    const uint8_t* hc1p = pick64(p, A.hc1);
    const uint8_t* hc2p = pick64(p, A.hc2);
    const uchar4 mc1 = *reinterpret_cast<const uchar4*>(hc1p + h0);
    const uchar4 mc2 = *reinterpret_cast<const uchar4*>(hc2p + h0);
    const uint8_t* cards = A.chance_cards + T.cards;
    for (uint32_t i = 0; i < T.nchild; i++) {
      if (A.alive[T.child_slot + i] == 0) continue;
      const uint8_t card = cards[i];
      double v[V64];
      ld4d(A.vals + (size_t)(T.child + i) * stride + h0, v);
#pragma unroll
      for (int j = 0; j < V64; j++) {
        const bool blocked = (&mc1.x)[j] == card || (&mc2.x)[j] == card;
        out[j] += blocked ? 0.0 : v[j];
      }
    }
    const int np = pick64(p, A.n);
    for (uint32_t k = 0; k < T.iso_count; k++) {
      const IsoRefD ref = A.iso[T.iso_first + k];
      if (A.alive[T.child_slot + ref.ci] == 0) continue;
      const uint8_t card = cards[ref.ci];
      const double* row = A.vals + (size_t)(T.child + ref.ci) * stride;
      const uint16_t* perm = A.perm + (size_t)(p * 6 + ref.pair) * stride;
#pragma unroll
      for (int j = 0; j < V64; j++) {
        const int h = h0 + j;
        if (h < np) {
          const int q = perm[h];
          const bool blocked = hc1p[q] == card || hc2p[q] == card;
          out[j] += blocked ? 0.0 : row[q];
        }
      }
    }
  }
  st4d(A.vals + (size_t)T.node * stride + h0, out);
}

__global__ void __launch_bounds__(ROW_MAX_THREADS) down64_kernel(Row64Args A, const DownTask* __restrict__ tasks,
                                                                 int chunks) {
  const int t = blockIdx.x / chunks, ch = blockIdx.x - t * chunks;
  const DownTask T = tasks[t];
  down64_item(A, T, (ch * (int)blockDim.x + (int)threadIdx.x) * V64, threadIdx.x & 31);
}

template <int MODE>
__global__ void __launch_bounds__(ROW_MAX_THREADS) up64_kernel(Row64Args A, const UpTask* __restrict__ tasks,
                                                               int chunks) {
  const int t = blockIdx.x / chunks, ch = blockIdx.x - t * chunks;
  const UpTask T = tasks[t];
  up64_item<MODE>(A, T, (ch * (int)blockDim.x + (int)threadIdx.x) * V64);
}

// One block per fused river subtree: its down tasks in BFS order (a barrier
// at every new level), then its up tasks deepest first. A thread keeps the
// same 4 hands, so each row is produced and consumed by the same thread
// except across the level barrier.
__global__ void __launch_bounds__(ROW_MAX_THREADS) fused_down64_kernel(Row64Args A, const FusedTree* __restrict__ trees,
                                                                       const DownTask* __restrict__ tasks) {
  const FusedTree F = trees[blockIdx.x];
  const int lane = threadIdx.x & 31;
  for (uint32_t i = 0; i < F.down_count; i++) {
    const DownTask T = tasks[F.down_first + i];
    if (T.kind & LEVEL_BREAK) __syncthreads();
    // The block covers the whole row in one pass (threads_for), and every
    // lane calls the item: it holds a warp vote.
    down64_item(A, T, (int)threadIdx.x * V64, lane);
  }
}

template <int MODE>
__global__ void __launch_bounds__(ROW_MAX_THREADS) fused_up64_kernel(Row64Args A, const FusedTree* __restrict__ trees,
                                                                     const UpTask* __restrict__ tasks) {
  const FusedTree F = trees[blockIdx.x];
  for (uint32_t i = 0; i < F.up_count; i++) {
    const UpTask T = tasks[F.up_first + i];
    up64_item<MODE>(A, T, (int)threadIdx.x * V64);
  }
}

int threads_for(int hp, int& chunks) {
  const int quads = (hp + V64 - 1) / V64;
  int threads = ((quads + 31) / 32) * 32;
  if (threads > ROW_MAX_THREADS) threads = ROW_MAX_THREADS;
  if (threads < 32) threads = 32;
  chunks = (quads + threads - 1) / threads;
  return threads;
}

}  // namespace

void launch_down64(const Row64Args& A, const DownTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (ntasks <= 0) return;
  int chunks = 1;
  const int threads = threads_for(hp, chunks);
  down64_kernel<<<ntasks * chunks, threads, 0, s>>>(A, tasks, chunks);
}

void launch_up64(int mode, const Row64Args& A, const UpTask* tasks, int ntasks, int hp, cudaStream_t s) {
  if (ntasks <= 0) return;
  int chunks = 1;
  const int threads = threads_for(hp, chunks);
  if (mode == M_BR) up64_kernel<M_BR><<<ntasks * chunks, threads, 0, s>>>(A, tasks, chunks);
  else up64_kernel<M_AVG><<<ntasks * chunks, threads, 0, s>>>(A, tasks, chunks);
}

void launch_fused_down64(const Row64Args& A, const FusedTree* trees, int ntrees, const DownTask* tasks,
                         cudaStream_t s) {
  if (ntrees <= 0) return;
  int chunks = 1;
  const int threads = threads_for(A.stride, chunks);
  fused_down64_kernel<<<ntrees, threads, 0, s>>>(A, trees, tasks);
}

void launch_fused_up64(int mode, const Row64Args& A, const FusedTree* trees, int ntrees, const UpTask* tasks,
                       cudaStream_t s) {
  if (ntrees <= 0) return;
  int chunks = 1;
  const int threads = threads_for(A.stride, chunks);
  if (mode == M_BR) fused_up64_kernel<M_BR><<<ntrees, threads, 0, s>>>(A, trees, tasks);
  else fused_up64_kernel<M_AVG><<<ntrees, threads, 0, s>>>(A, trees, tasks);
}

}  // namespace dcfr
