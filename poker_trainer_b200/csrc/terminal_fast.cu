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

namespace dcfr {

namespace {

__device__ __forceinline__ double pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

// Fixed-point value of one reach entry: trunc(x * 2^S). Products are exact
// (power-of-two scale, below 2^52).
__device__ __forceinline__ long long fixed(float x, double scale) { return __double2ll_rz((double)x * scale); }

}  // namespace

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

// One block per task at a time (grid-stride over the task list).
__global__ void __launch_bounds__(FAST_THREADS) fast_terminal_kernel(FastArgs A, const FastTask* __restrict__ tasks,
                                                                     int ntasks) {
  extern __shared__ __align__(16) unsigned char smem_fast[];
  const int E = A.emax;
  const int gn = (FAST_THREADS * E + 2) & ~1;
  float* r = reinterpret_cast<float*>(smem_fast);
  long long* G = reinterpret_cast<long long*>(r + A.stride);
  long long* Cs = G + gn;
  long long* wsum = Cs + FAST_SEGS;
  float* fred = reinterpret_cast<float*>(wsum + FAST_THREADS / 32);

  const int p = A.p, o = p ^ 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int hpo = o ? A.hp[1] : A.hp[0], hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  for (int ti = blockIdx.x; ti < ntasks; ti += gridDim.x) {
    const FastTask& T = tasks[ti];
    const uint32_t slot = T.slot;
    if (A.alive[slot] == 0) continue;  // dead subtree (cfr.rs:267-274): row untouched
    const size_t lay = (size_t)T.board * 2 + p;
    const uint16_t* seg = A.seg + lay * FAST_SEGS;
    const int L = seg[FAST_SEGS - 1];

    // Reach row into shared memory, and its maximum.
    const float4* src = reinterpret_cast<const float4*>(A.reach + (size_t)slot * A.stride);
    float mx = 0.0f;
    for (int i = tid; i < hpo / 4; i += FAST_THREADS) {
      const float4 v = src[i];
      reinterpret_cast<float4*>(r)[i] = v;
      mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, d));
    if (lane == 0) fred[warp] = mx;
    __syncthreads();
#pragma unroll
    for (int w = 0; w < FAST_THREADS / 32; w++) mx = fmaxf(mx, fred[w]);
    // Row sum < 2048 * 2^(e+1) with 2^e <= max: scale it below 2^62.
    const int S = 177 - (int)((__float_as_uint(mx) >> 23) & 0xFF);
    const double scale = pow2(S), inv = pow2(-S);

    // Elements in layout order, as fixed point.
    const uint16_t* cat = A.cat + lay * A.cstride;
    for (int k = tid; k < FAST_THREADS * E; k += FAST_THREADS) G[k] = k < L ? fixed(r[cat[k]], scale) : 0;
    __syncthreads();

    // Exclusive prefix sums, in place: E consecutive elements per thread.
    long long* own = G + tid * E;
    long long local = 0;
    for (int i = 0; i < E; i++) local += own[i];
    long long inc = local;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    long long acc = inc - local;
    for (int w = 0; w < warp; w++) acc += wsum[w];
    for (int i = 0; i < E; i++) {
      const long long x = own[i];
      own[i] = acc;
      acc += x;
    }
    if (tid == FAST_THREADS - 1) G[FAST_THREADS * E] = acc;
    __syncthreads();
    if (tid < FAST_SEGS) Cs[tid] = G[seg[tid]];
    __syncthreads();

    // Values in hand order.
    const uint4* rec = A.rec + lay * A.tstride;
    const long long T0 = Cs[1];
    float* out = A.vals + (size_t)T.row * A.stride;
    const uint32_t frow = T.frow, kind = T.kind;
    float* fout = frow != NONE32 ? A.vals + (size_t)frow * A.stride : nullptr;
    const bool fold = kind == T_FOLD_SCALAR || kind == T_FOLD_BATCH;
    const bool scalar = kind == T_FOLD_SCALAR || kind == T_SHOWDOWN_SCALAR;
    const double pa = T.a, pb = T.b, pc = T.c, pd = T.d;
    for (int h = tid; h < hpp; h += FAST_THREADS) {
      float v = 0.0f, fv = 0.0f;
      if (h < np) {
        const uint4 q = rec[h];
        const int a = q.w & 0xFF, b = (q.w >> 8) & 0xFF;
        const long long C0a = Cs[1 + a], CTa = Cs[2 + a] - C0a;
        const long long C0b = Cs[1 + b], CTb = Cs[2 + b] - C0b;
        const uint32_t sm = A.same[h];
        const long long si = sm != NONE32 ? fixed(r[sm], scale) : 0;
        const long long F = T0 - CTa - CTb + si;
        if (fold) {
          // eval_fold (eval.rs:40-64) returns zeros on a zero total.
          v = (scalar && T0 == 0) ? 0.0f : (float)(pa * ((double)F * inv));
        } else {
          if (q.w >> 16) {
            const long long Gw = G[q.x & 0xFFFF], Gs = G[q.x >> 16];
            const long long Ca = G[q.y & 0xFFFF] - C0a, Cal = G[q.y >> 16] - C0a;
            const long long Cb = G[q.z & 0xFFFF] - C0b, Cbl = G[q.z >> 16] - C0b;
            const double fw = (double)(Gw - Ca - Cb) * inv;
            const double fl = (double)((T0 - Gs) - (CTa - Cal) - (CTb - Cbl)) * inv;
            if (scalar) {
              v = (float)(pa * fw) + (float)(pb * fl);
            } else {
              double res = pa * fw;
              res += pb * fl;
              v = (float)res;
            }
            if (pc != 0.0) {
              const long long eq = (Gs - Gw) - (Cal - Ca) - (Cbl - Cb) + si;
              v += (float)(pc * ((double)eq * inv));
            }
          }
          fv = (float)(pd * ((double)F * inv));
        }
      }
      out[h] = v;
      if (fout) fout[h] = fv;
    }
    __syncthreads();
  }
}

int fast_emax(int tstride) {
  const int e = (3 * tstride + FAST_THREADS - 1) / FAST_THREADS;
  return e | 1;  // odd: conflict-free strided f64 access
}

size_t fast_smem_bytes(int stride, int emax) {
  const int gn = (FAST_THREADS * emax + 2) & ~1;
  return (size_t)stride * 4 + (size_t)gn * 8 + FAST_SEGS * 8 + (FAST_THREADS / 32) * 8 + (FAST_THREADS / 32) * 4;
}

int fast_blocks_per_sm(int stride, int emax) {
  int blocks = 0;
  const size_t smem = fast_smem_bytes(stride, emax);
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(fast_terminal_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fast_terminal_kernel, FAST_THREADS, smem) != cudaSuccess)
    return 1;
  return blocks > 0 ? blocks : 1;
}

void launch_fast_layouts(const EntryD* tables, const uint32_t* count, int tstride, int nboards, const uint8_t* hc1_0,
                         const uint8_t* hc2_0, const uint8_t* hc1_1, const uint8_t* hc2_1, int n0, int n1,
                         uint16_t* cat, uint16_t* seg, uint4* rec, int cstride, cudaStream_t s) {
  const int n = (nboards + 1) * 2;
  fast_layout_kernel<<<(n + 63) / 64, 64, 0, s>>>(tables, count, tstride, nboards, hc1_0, hc2_0, hc1_1, hc2_1, n0, n1,
                                                  cat, seg, rec, cstride);
}

void launch_fast_terminal(const FastArgs& A, const FastTask* tasks, int ntasks, int max_blocks, cudaStream_t s) {
  if (ntasks <= 0) return;
  const int blocks = ntasks < max_blocks ? ntasks : max_blocks;
  fast_terminal_kernel<<<blocks, FAST_THREADS, fast_smem_bytes(A.stride, A.emax), s>>>(A, tasks, ntasks);
}

}  // namespace dcfr
