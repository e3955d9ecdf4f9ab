// Leaf evaluation of depth-limited solves. A depth-limited flop solve ends
// its tree at the turn deal (N_LEAF nodes); every traversal values those
// leaves with the leaf-value network instead of the turn and river subtrees:
//
//   capture: the opponent's reach arriving at each leaf is kept per player
//            (the network takes both players' ranges; the traverser's own
//            range is the one its opponent's latest traversal delivered);
//   inputs:  one network row per (leaf, dealt card): both ranges in combo
//            order with the hands holding the card removed, scaled to a
//            maximum of 1, the board and dealt card one-hot, pot and stack;
//   values:  the network gives every combo's EV (in pots) after that card;
//            the leaf's counterfactual value of traverser hand h is
//              norm * factor * pot * sum_c [c not in h] EV_c(h) * m_c(h),
//            the same sum a chance node forms over its children
//            (cfr.rs:435-479), after a zero-sum correction of each card's
//            network values (see leaf_values_kernel), where m_c(h) is the
//            opponent reach
//            compatible with h and c: with T the total, A[x] the reach of
//            hands holding card x and R{x,y} the reach of combo {x,y},
//              m_c(h) = T - A[h1] - A[h2] + R{h1,h2} - (A[c] - R{c,h1} - R{c,h2}).
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.hpp"

namespace dcfr {

namespace {

constexpr int LEAF_IN = 2 * DCFR_NUM_COMBOS + 52 + 2;
constexpr float LEAF_SCALE = 10000.0f;

__device__ __forceinline__ int combo_of(int a, int b) {
  const int hi = a > b ? a : b, lo = a > b ? b : a;
  return hi * (hi - 1) / 2 + lo;
}

__global__ void leaf_capture_kernel(LeafArgs A, const LeafTask* __restrict__ tasks) {
  const LeafTask T = tasks[blockIdx.x];
  const int o = A.p ^ 1;
  float* dst = A.leaf_reach[o] + (size_t)T.leaf * A.stride;
  const float* src = A.reach + (size_t)T.slot * A.stride;
  const bool live = A.alive[T.slot] != 0;
  for (int h = threadIdx.x; h < A.stride; h += blockDim.x) dst[h] = live ? src[h] : 0.0f;
}

// Block (leaf task, card index): one input row.
__global__ void leaf_inputs_kernel(LeafArgs A, const LeafTask* __restrict__ tasks, const uint8_t* __restrict__ hc1_0,
                                   const uint8_t* __restrict__ hc2_0, const uint8_t* __restrict__ hc1_1,
                                   const uint8_t* __restrict__ hc2_1) {
  const LeafTask T = tasks[blockIdx.x];
  const int ci = blockIdx.y;
  const int card = A.cards[ci];
  float* x = A.x + ((size_t)T.leaf * A.nc + ci) * LEAF_IN;
  __shared__ float red[32];
  for (int i = threadIdx.x; i < LEAF_IN; i += blockDim.x) x[i] = 0.0f;
  __syncthreads();
  for (int q = 0; q < 2; q++) {
    const float* r = A.leaf_reach[q] + (size_t)T.leaf * A.stride;
    const uint8_t* c1 = q ? hc1_1 : hc1_0;
    const uint8_t* c2 = q ? hc2_1 : hc2_0;
    const uint16_t* cb = A.combos[q];
    float mx = 0.0f;
    for (int h = threadIdx.x; h < A.n[q]; h += blockDim.x)
      if (c1[h] != card && c2[h] != card) mx = fmaxf(mx, r[h]);
    for (int d = 16; d > 0; d >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    mx = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) mx = fmaxf(mx, red[w]);
    const float inv = mx > 0.0f ? 1.0f / mx : 0.0f;
    for (int h = threadIdx.x; h < A.n[q]; h += blockDim.x)
      x[q * DCFR_NUM_COMBOS + cb[h]] = (c1[h] != card && c2[h] != card) ? r[h] * inv : 0.0f;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < 3; k++) x[2 * DCFR_NUM_COMBOS + A.board[k]] = 1.0f;
    x[2 * DCFR_NUM_COMBOS + card] = 1.0f;
    x[2 * DCFR_NUM_COMBOS + 52] = T.pot / LEAF_SCALE;
    x[2 * DCFR_NUM_COMBOS + 53] = T.stack / LEAF_SCALE;
  }
}

// Block per leaf task: the traverser's value row at the leaf. Before the
// sum, each card's network values are made zero-sum (as the subgame is):
// with S_q = sum over q's hands of r_q(h) m_c(h) EV_q,c(h) and M the joint
// compatible mass, both sides are shifted by (S_p + S_o) / (2 M), so the
// corrected values satisfy S_p + S_o = 0 exactly.
__global__ void leaf_values_kernel(LeafArgs A, const LeafTask* __restrict__ tasks, const uint8_t* __restrict__ hc1_p,
                                   const uint8_t* __restrict__ hc2_p, const uint8_t* __restrict__ hc1_o,
                                   const uint8_t* __restrict__ hc2_o, int hp) {
  const LeafTask T = tasks[blockIdx.x];
  if (A.alive[T.slot] == 0) return;  // dead subtree (cfr.rs:267-274): row untouched
  const int p = A.p, o = p ^ 1;
  __shared__ float R[2][DCFR_NUM_COMBOS];  // [0]: opponent, [1]: traverser, combo order
  __shared__ double Acard[2][52];
  __shared__ double total[2];
  __shared__ double red[3][32];
  __shared__ double shift[64];
  const float* ro = A.reach + (size_t)T.slot * A.stride;
  const float* rp = A.leaf_reach[p] + (size_t)T.leaf * A.stride;
  for (int i = threadIdx.x; i < 2 * DCFR_NUM_COMBOS; i += blockDim.x) (&R[0][0])[i] = 0.0f;
  for (int i = threadIdx.x; i < 104; i += blockDim.x) (&Acard[0][0])[i] = 0.0;
  if (threadIdx.x < 2) total[threadIdx.x] = 0.0;
  __syncthreads();
  for (int side = 0; side < 2; side++) {
    const int q = side ? p : o;
    const float* r = side ? rp : ro;
    const uint8_t* c1 = side ? hc1_p : hc1_o;
    const uint8_t* c2 = side ? hc2_p : hc2_o;
    const uint16_t* cb = A.combos[q];
    for (int j = threadIdx.x; j < A.n[q]; j += blockDim.x) {
      const float v = r[j];
      R[side][cb[j]] = v;
      if (v != 0.0f) {
        atomicAdd(&Acard[side][c1[j]], (double)v);
        atomicAdd(&Acard[side][c2[j]], (double)v);
        atomicAdd(&total[side], (double)v);
      }
    }
  }
  __syncthreads();
  // m_c for a hand of one side: the other side's reach compatible with it and c.
  auto mass = [&](int other, int h1, int h2, int ch, int c) -> double {
    return total[other] - Acard[other][h1] - Acard[other][h2] + (double)R[other][ch] -
           (Acard[other][c] - (double)R[other][combo_of(c, h1)] - (double)R[other][combo_of(c, h2)]);
  };
  const float* ybase = A.y + (size_t)T.leaf * A.nc * A.ldy;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int ci = 0; ci < A.nc; ci++) {
    const int c = A.cards[ci];
    const float* y = ybase + (size_t)ci * A.ldy;
    double sp = 0.0, so = 0.0, mm = 0.0;
    for (int h = threadIdx.x; h < A.n[p]; h += blockDim.x) {
      const int h1 = hc1_p[h], h2 = hc2_p[h];
      if (h1 == c || h2 == c) continue;
      const int ch = A.combos[p][h];
      const double w = (double)R[1][ch] * mass(0, h1, h2, ch, c);
      sp += w * (double)y[(size_t)p * DCFR_NUM_COMBOS + ch];
      mm += w;
    }
    for (int j = threadIdx.x; j < A.n[o]; j += blockDim.x) {
      const int h1 = hc1_o[j], h2 = hc2_o[j];
      if (h1 == c || h2 == c) continue;
      const int ch = A.combos[o][j];
      so += (double)R[0][ch] * mass(1, h1, h2, ch, c) * (double)y[(size_t)o * DCFR_NUM_COMBOS + ch];
    }
    for (int d = 16; d > 0; d >>= 1) {
      sp += __shfl_xor_sync(0xffffffffu, sp, d);
      so += __shfl_xor_sync(0xffffffffu, so, d);
      mm += __shfl_xor_sync(0xffffffffu, mm, d);
    }
    if (lane == 0) {
      red[0][warp] = sp;
      red[1][warp] = so;
      red[2][warp] = mm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0, m = 0.0;
      for (int w = 0; w < nw; w++) {
        a += red[0][w];
        b += red[1][w];
        m += red[2][w];
      }
      shift[ci] = m > 0.0 ? 0.5 * (a + b) / m : 0.0;
    }
    __syncthreads();
  }
  float* out = A.vals + (size_t)T.row * A.stride;
  const double scale = A.norm * (double)A.factor * (double)T.pot;
  for (int h = threadIdx.x; h < hp; h += blockDim.x) {
    float v = 0.0f;
    if (h < A.n[p]) {
      const int h1 = hc1_p[h], h2 = hc2_p[h];
      const int ch = A.combos[p][h];
      double acc = 0.0;
      for (int ci = 0; ci < A.nc; ci++) {
        const int c = A.cards[ci];
        if (c == h1 || c == h2) continue;
        const double ev = (double)ybase[(size_t)ci * A.ldy + (size_t)p * DCFR_NUM_COMBOS + ch] - shift[ci];
        acc += ev * mass(0, h1, h2, ch, c);
      }
      v = (float)(scale * acc);
    }
    out[h] = v;
  }
}

}  // namespace

void launch_leaf_capture(const LeafArgs& A, const LeafTask* tasks, int ntasks, cudaStream_t s) {
  if (ntasks > 0) leaf_capture_kernel<<<ntasks, 128, 0, s>>>(A, tasks);
}

void launch_leaf_inputs(const LeafArgs& A, const LeafTask* tasks, int ntasks, const uint8_t* hc1_0,
                        const uint8_t* hc2_0, const uint8_t* hc1_1, const uint8_t* hc2_1, cudaStream_t s) {
  if (ntasks > 0) leaf_inputs_kernel<<<dim3(ntasks, A.nc), 256, 0, s>>>(A, tasks, hc1_0, hc2_0, hc1_1, hc2_1);
}

void launch_leaf_values(const LeafArgs& A, const LeafTask* tasks, int ntasks, const uint8_t* hc1_p,
                        const uint8_t* hc2_p, const uint8_t* hc1_o, const uint8_t* hc2_o, int hp, cudaStream_t s) {
  if (ntasks > 0) leaf_values_kernel<<<ntasks, 256, 0, s>>>(A, tasks, hc1_p, hc2_p, hc1_o, hc2_o, hp);
}

}  // namespace dcfr
