// Panel terminal evaluation: the fast-precision terminal kernel of the solve
// (f32 rows).
//
// It computes what fast_terminal_kernel and warp_terminal_kernel compute
// (terminal_fast.cu, warp_terminal.cuh): every fold and showdown value of
// the reference's evaluators (crates/solver/src/eval.rs:40-379) from exact
// 64-bit fixed-point prefix sums over a board's scan layout, with the same
// integer sums and the same final f64/f32 operations, so its results are
// bit-identical to theirs.
//
// What changes is the shape of the work. A panel is up to T terminals of
// one layout (one river board, or the fold layout). A block evaluates a
// panel's T terminals together:
//   - the T reach rows are staged row-major with a padded stride, so the T
//     lanes that gather one layout element read T different banks;
//   - the prefix array is interleaved [element][T]: lane t of a group of T
//     lanes works on terminal t, and the T lanes that look up one position
//     read T consecutive 8-byte prefixes instead of T scattered ones;
//   - the layout (elements, per-hand records, segment starts) and every
//     per-hand record read is shared by the T terminals.
// A random 8-byte gather by 32 lanes costs several shared-memory wavefronts
// (bank conflicts); 32/T random gathers of T x 8 contiguous bytes cost
// close to the minimum. The scan keeps each thread's E layout elements in
// registers between its two passes, so the prefix array is written once.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"
#include "warp_terminal.cuh"

namespace dcfr {

constexpr int PANEL_THREADS = 512;
constexpr int PANEL_WARPS = PANEL_THREADS / 32;

// Shared-memory layout of a block (every offset 16-byte aligned). E x
// (threads / T) scan positions: the layout padded past its end, so the scan
// needs no bounds test.
struct PanelSmem {
  size_t rows, g, cat, rec, same, seg, pairs, t0, wsum, wmax, task, alive, total;
  int rstride;  // floats per staged row: hpo + 4 (16-byte rows; bank stagger)
  int npos;     // scan positions
  __host__ __device__ PanelSmem(int hpo, int hpp, int tstride, int T, int E) {
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    rstride = hpo + 4;
    npos = E * (PANEL_THREADS / T);
    rows = 0;                                                  // [2][T][rstride] f32
    g = up16(rows + (size_t)2 * T * rstride * 4);              // [npos][T] i64
    cat = up16(g + (size_t)npos * T * 8);                      // [npos] u16
    rec = up16(cat + (size_t)npos * 2);                        // [tstride] uint4
    same = up16(rec + (size_t)tstride * 16);                   // [hpp] u16
    seg = up16(same + (size_t)hpp * 2);                        // [FAST_SEGS] u16
    pairs = up16(seg + FAST_SEGS * 2);                         // [52][T] {prefix at card segment start, at end}
    t0 = up16(pairs + (size_t)52 * T * 16);                    // [T] i64: the main segment's total
    wsum = up16(t0 + (size_t)T * 8);                           // [PANEL_WARPS][T] i64
    wmax = up16(wsum + (size_t)PANEL_WARPS * T * 8);           // [2][T][PANEL_WARPS] f32 row-maximum partials
    task = up16(wmax + (size_t)2 * T * PANEL_WARPS * 4);       // [3][T] FastTask (ring)
    alive = up16(task + (size_t)3 * T * sizeof(FastTask));     // [2][T] u32
    total = up16(alive + (size_t)2 * T * 4);
  }
};

__device__ __forceinline__ void panel_cp16(void* dst, const void* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// One block per SM. Block b takes the contiguous panel range
// [b N / G, (b+1) N / G) (panels are ordered by layout) and stages a
// layout when its range enters it. Per panel, three block barriers:
//   (A) the previous panel is done; this panel's rows, row-maximum partials,
//       liveness flags and the next panel's task records are in place;
//   (C) per-warp scan totals written;
//   (D) prefixes and segment-boundary prefixes written;
// and one more where a new layout is staged. Nothing on the way waits for
// global memory: task records come through a three-panel ring of
// asynchronous copies, the next panel's rows are copied while this one
// runs, and at the end of a panel every thread waits for its own copies of
// the next rows and reduces their maxima (each thread reads only what it
// copied), so the next panel starts with its scales ready.
template <int T, int E>
__global__ void __launch_bounds__(PANEL_THREADS, 1)
    panel_terminal_kernel(FastArgs A, const FastTask* __restrict__ tasks, const PanelD* __restrict__ panels,
                          int npanels) {
  extern __shared__ __align__(16) unsigned char smem_panel[];
  const int p = A.p, o = p ^ 1;
  const int hpo = o ? A.hp[1] : A.hp[0], hpp = p ? A.hp[1] : A.hp[0], np = p ? A.n[1] : A.n[0];
  const PanelSmem Ls(hpo, hpp, A.tstride, T, E);
  float* rows = reinterpret_cast<float*>(smem_panel + Ls.rows);
  long long* G = reinterpret_cast<long long*>(smem_panel + Ls.g);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_panel + Ls.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_panel + Ls.rec);
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_panel + Ls.same);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_panel + Ls.seg);
  longlong2* pairs = reinterpret_cast<longlong2*>(smem_panel + Ls.pairs);
  long long* pairs_ll = reinterpret_cast<long long*>(smem_panel + Ls.pairs);
  long long* st0 = reinterpret_cast<long long*>(smem_panel + Ls.t0);
  long long* wsum = reinterpret_cast<long long*>(smem_panel + Ls.wsum);
  float* wmax = reinterpret_cast<float*>(smem_panel + Ls.wmax);
  FastTask* ring = reinterpret_cast<FastTask*>(smem_panel + Ls.task);
  uint32_t* salive = reinterpret_cast<uint32_t*>(smem_panel + Ls.alive);
  const int rstride = Ls.rstride, npos = Ls.npos;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t = lane % T;                          // this thread's terminal within a panel
  constexpr int CPW = 32 / T;                      // scan chunks per warp
  const int k0 = (warp * CPW + lane / T) * E;      // first layout position of this thread's chunk
  constexpr int HSTEP = PANEL_THREADS / T;         // hands per value pass
  constexpr int TWORDS = (int)(sizeof(FastTask) / 16);
  const int per = hpo >> 2;                        // 16-byte chunks per row

  const int b0 = (int)(((long long)blockIdx.x * npanels) / gridDim.x);
  const int b1 = (int)(((long long)(blockIdx.x + 1) * npanels) / gridDim.x);
  if (b0 >= b1) return;

  for (int h = tid; h < hpp; h += PANEL_THREADS) {
    const uint32_t sm = h < np ? A.same[h] : NONE32;
    ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
  }
  // Task records of panel pi into ring entry r (16-byte copies).
  auto fetch_tasks = [&](int pi, int r) {
    const PanelD P = panels[pi];
    if (tid < (int)P.count * TWORDS) {
      const int tt = tid / TWORDS, w = tid - tt * TWORDS;
      panel_cp16(reinterpret_cast<unsigned char*>(ring + r * T + tt) + 16 * w,
                 reinterpret_cast<const unsigned char*>(tasks + P.first + tt) + 16 * w);
    }
  };
  // Rows of panel pi (task records in ring entry r) into buffer b: thread
  // tid copies chunks j = tid, tid + threads, ... of every row.
  auto fetch_rows = [&](int pi, int r, int b) {
    const int cnt = (int)panels[pi].count;
    float* dst = rows + (size_t)b * T * rstride;
#pragma unroll
    for (int tt = 0; tt < T; tt++)
      if (tt < cnt) {
        const float* src = A.reach + (size_t)ring[r * T + tt].slot * A.stride;
        for (int j = tid; j < per; j += PANEL_THREADS) panel_cp16(dst + (size_t)tt * rstride + 4 * j, src + 4 * j);
      }
  };
  // Per-warp maxima of the rows of panel pi in buffer b, from the chunks
  // this thread copied, after its own cp.async wait: wmax[b][row][warp].
  auto own_row_max = [&](int pi, int b) {
    const int cnt = (int)panels[pi].count;
    const float* src = rows + (size_t)b * T * rstride;
#pragma unroll
    for (int tt = 0; tt < T; tt++) {
      float m = 0.0f;
      if (tt < cnt)
        for (int j = tid; j < per; j += PANEL_THREADS) {
          const float4 v = *reinterpret_cast<const float4*>(src + (size_t)tt * rstride + 4 * j);
          m = fmaxf(m, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
        }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, d));
      if (lane == 0) wmax[(b * T + tt) * PANEL_WARPS + warp] = m;
    }
  };
  // Prologue: task records of the first two panels, then the first rows
  // and their maxima.
  fetch_tasks(b0, 0);
  if (b0 + 1 < b1) fetch_tasks(b0 + 1, 1);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  if (tid < (int)panels[b0].count) salive[tid] = A.alive[ring[tid].slot];
  fetch_rows(b0, 0, 0);
  cp_async_commit();
  cp_async_wait<0>();
  own_row_max(b0, 0);
  uint32_t layout = NONE32;
  int bfirst = 1;  // first segment boundary at or after this thread's chunk

  for (int pi = b0; pi < b1; pi++) {
    const int buf = (pi - b0) & 1, r = (pi - b0) % 3;
    __syncthreads();  // (A)
    // The panel after next's task records, the next panel's rows, and the
    // next panel's liveness flags (stored at the end of this panel).
    uint32_t next_alive = 0;
    if (pi + 1 < b1) {
      if (pi + 2 < b1) fetch_tasks(pi + 2, (r + 2) % 3);
      fetch_rows(pi + 1, (r + 1) % 3, buf ^ 1);
      if (tid < (int)panels[pi + 1].count) next_alive = A.alive[ring[((r + 1) % 3) * T + tid].slot];
    }
    cp_async_commit();
    const PanelD P = panels[pi];
    const float* rbase = rows + (size_t)buf * T * rstride;
    if (P.layout != layout) {  // block-uniform
      layout = P.layout;
      const size_t lay = (size_t)layout * 2 + p;
      const uint16_t* gseg = A.seg + lay * FAST_SEGS;
      if (tid < FAST_SEGS) sseg[tid] = gseg[tid];
      const int Ln = gseg[FAST_SEGS - 1];
      const uint16_t* gcat = A.cat + lay * A.cstride;
      // Positions past the layout's end read hand 0: their sums only reach
      // prefixes beyond the end, which nothing reads.
      for (int k = tid; k < npos; k += PANEL_THREADS) scat[k] = k < Ln ? gcat[k] : (uint16_t)0;
      const uint4* grec = A.rec + lay * A.tstride;
      for (int h = tid; h < np; h += PANEL_THREADS) srec[h] = grec[h];
      __syncthreads();  // the new layout is staged
      bfirst = 1;
      while (bfirst < FAST_SEGS && (int)sseg[bfirst] < k0) bfirst++;
    }
    // This thread's task (lane t of the panel).
    const bool has = t < (int)P.count;
    const FastTask& tk = ring[r * T + (has ? t : 0)];
    const bool live = has && salive[buf * T + t] != 0;
    float mx = 0.0f;
#pragma unroll
    for (int w = 0; w < PANEL_WARPS; w++) mx = fmaxf(mx, wmax[(buf * T + t) * PANEL_WARPS + w]);
    const int S = scale_exponent(mx);
    const double scale = pow2(S), inv = pow2(-S);
    const float* myrow = rbase + (size_t)t * rstride;

    // Scan: E consecutive positions per thread, held in registers.
    long long x[E];
    long long local = 0;
#pragma unroll
    for (int i = 0; i < E; i++) {
      x[i] = fixed(myrow[scat[k0 + i]], scale);
      local += x[i];
    }
    long long inc = local;
#pragma unroll
    for (int d = T; d < 32; d <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, inc, d);
      if (lane >= d) inc += y;
    }
    if (lane >= 32 - T) wsum[warp * T + t] = inc;
    __syncthreads();  // (C)
    // The totals of the warps before this one, for this lane's terminal:
    // lane l reads entries l, l + 32, ... ([warp][T], so all of terminal
    // l % T), then the lanes of one terminal sum theirs.
    long long before = 0;
#pragma unroll
    for (int q = 0; q < PANEL_WARPS * T / 32; q++) {
      const int idx = lane + 32 * q;
      if (idx / T < warp) before += wsum[idx];
    }
#pragma unroll
    for (int d = T; d < 32; d <<= 1) before += __shfl_xor_sync(0xffffffffu, before, d);
    long long acc = inc - local + before;
#pragma unroll
    for (int i = 0; i < E; i++) {
      G[(size_t)(k0 + i) * T + t] = acc;
      acc += x[i];
    }
    // Segment boundaries inside this chunk (read back from this thread's own
    // prefixes): card c's segment runs from boundary 1 + c to 2 + c, and
    // boundary 1 closes the main segment.
    for (int b = bfirst; b < FAST_SEGS; b++) {
      const int kb = sseg[b];
      if (kb >= k0 + E) break;
      const long long pb = G[(size_t)kb * T + t];
      if (b == 1) st0[t] = pb;
      if (b <= 52) pairs_ll[((b - 1) * T + t) * 2] = pb;
      if (b >= 2) pairs_ll[((b - 2) * T + t) * 2 + 1] = pb;
    }
    __syncthreads();  // (D)

    if (live) {
      const uint32_t kind = tk.kind;
      const bool fold = kind == T_FOLD_SCALAR || kind == T_FOLD_BATCH;
      const bool scalar = kind == T_FOLD_SCALAR || kind == T_SHOWDOWN_SCALAR;
      const double pa = tk.a * inv, pb = tk.b * inv, pc = tk.c * inv, pd = tk.d * inv;
      const bool tie = tk.c != 0.0;
      const long long T0 = st0[t];
      float* out = A.vals + (size_t)tk.row * A.stride;
      float* fout = tk.frow != NONE32 ? A.vals + (size_t)tk.frow * A.stride : nullptr;
      const long long* Gt = G + t;
      auto value = [&](int h, float& v, float& fv) {
        v = 0.0f;
        fv = 0.0f;
        if (h >= np) return;
        const uint4 q = srec[h];
        const int a = (int)(q.w & 0xFF), bb = (int)((q.w >> 8) & 0xFF);
        // Card a's segment: prefix at its start (sa) and end (ea).
        const longlong2 ca = pairs[a * T + t], cb = pairs[bb * T + t];
        const long long sab = ca.x + cb.x, base = T0 - (ca.y + cb.y);
        const uint16_t sm = ssame[h];
        const long long si = sm == 0xFFFF ? 0ll : fixed(myrow[sm], scale);
        // fold: T - (card a total) - (card b total) + identical hand.
        const long long F = base + sab + si;
        if (fold) {
          // eval_fold (eval.rs:40-64) returns zeros on a zero total.
          v = (scalar && T0 == 0) ? 0.0f : (float)(pa * (double)F);
          return;
        }
        if (q.w >> 16) {
          const long long Gw = Gt[(q.x & 0xFFFF) * T], Gs = Gt[(q.x >> 16) * T];
          const long long Gaw = Gt[(q.y & 0xFFFF) * T], Gas = Gt[(q.y >> 16) * T];
          const long long Gbw = Gt[(q.z & 0xFFFF) * T], Gbs = Gt[(q.z >> 16) * T];
          // weaker: Gw - (Gaw - sa) - (Gbw - sb); stronger: (T0 - Gs)
          // - (ea - Gas) - (eb - Gbs).
          const long long Wn = (Gw + sab) - Gaw - Gbw;
          const long long Lx = (base + Gas + Gbs) - Gs;
          if (scalar) {
            v = (float)(pa * (double)Wn) + (float)(pb * (double)Lx);
          } else {
            double res = pa * (double)Wn;
            res += pb * (double)Lx;
            v = (float)res;
          }
          if (tie) {
            const long long eq = (Gs - Gw) - (Gas - Gaw) - (Gbs - Gbw) + si;
            v += (float)(pc * (double)eq);
          }
        }
        if (fout) fv = (float)(pd * (double)F);
      };
      // Two hands per step: both hands' loads are issued before the stores.
      int h = tid / T;
      for (; h + HSTEP < hpp; h += 2 * HSTEP) {
        float v0, f0, v1, f1;
        value(h, v0, f0);
        value(h + HSTEP, v1, f1);
        out[h] = v0;
        out[h + HSTEP] = v1;
        if (fout) {
          fout[h] = f0;
          fout[h + HSTEP] = f1;
        }
      }
      for (; h < hpp; h += HSTEP) {
        float v0, f0;
        value(h, v0, f0);
        out[h] = v0;
        if (fout) fout[h] = f0;
      }
    }
    // Dead subtree (cfr.rs:267-274) or no task: rows untouched.
    // The next panel: its rows (this thread's copies) and their maxima, and
    // its liveness flags.
    cp_async_wait<0>();
    if (pi + 1 < b1) {
      own_row_max(pi + 1, buf ^ 1);
      if (tid < (int)panels[pi + 1].count) salive[(buf ^ 1) * T + tid] = next_alive;
    }
  }
  cp_async_wait<0>();
}

// Elements per thread of the instantiated kernels (odd: a thread's 8-byte
// prefixes of consecutive chunks fall on different banks).
#define PANEL_ES(X) X(7) X(11) X(15) X(19) X(23) X(27) X(31)

static int panel_e_for(int cstride, int T) {
  const int chunks = PANEL_THREADS / T;
#define PANEL_PICK(e_) \
  if ((e_) * chunks >= cstride + 1) return e_;
  PANEL_ES(PANEL_PICK)
#undef PANEL_PICK
  return 0;
}

size_t panel_terminal_smem(int hpo, int hpp, int cstride, int tstride, int T) {
  return PanelSmem(hpo, hpp, tstride, T, panel_e_for(cstride, T)).total;
}

template <int T>
static const void* panel_fn(int e) {
  switch (e) {
#define PANEL_CASE(e_) \
  case e_:             \
    return (const void*)panel_terminal_kernel<T, e_>;
    PANEL_ES(PANEL_CASE)
#undef PANEL_CASE
  }
  return nullptr;
}

static const void* panel_kernel(int T, int e) { return T == 8 ? panel_fn<8>(e) : T == 4 ? panel_fn<4>(e) : nullptr; }

// Sets the kernel's shared-memory limit for terminals of T lanes; returns
// the elements per thread (0 if the layout does not fit) and the blocks per
// SM.
int panel_terminal_setup(int hpo, int hpp, int cstride, int tstride, int T, int& blocks_per_sm) {
  blocks_per_sm = 0;
  const int e = panel_e_for(cstride, T);
  const void* fn = panel_kernel(T, e);
  if (!fn) return 0;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  const size_t smem = panel_terminal_smem(hpo, hpp, cstride, tstride, T);
  if (smem > (size_t)optin) return 0;
  // The limit is the device's opt-in maximum (a per-kernel setting shared by
  // every handle and both traversers), not this footprint.
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess) return 0;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, PANEL_THREADS, smem) != cudaSuccess || b <= 0) return 0;
  blocks_per_sm = b;
  return e;
}

void launch_panel_terminal(const FastArgs& A, const FastTask* tasks, const PanelD* panels, int npanels, int T, int e,
                           int max_blocks, cudaStream_t s) {
  if (npanels <= 0) return;
  const int hpo = A.hp[A.p ^ 1], hpp = A.hp[A.p];
  const size_t smem = panel_terminal_smem(hpo, hpp, A.cstride, A.tstride, T);
  const int blocks = npanels < max_blocks ? npanels : max_blocks;
  if (T == 8) {
    switch (e) {
#define PANEL_L8(e_)                                                                              \
  case e_:                                                                                        \
    panel_terminal_kernel<8, e_><<<blocks, PANEL_THREADS, smem, s>>>(A, tasks, panels, npanels); \
    break;
      PANEL_ES(PANEL_L8)
#undef PANEL_L8
    }
  } else {
    switch (e) {
#define PANEL_L4(e_)                                                                              \
  case e_:                                                                                        \
    panel_terminal_kernel<4, e_><<<blocks, PANEL_THREADS, smem, s>>>(A, tasks, panels, npanels); \
    break;
      PANEL_ES(PANEL_L4)
#undef PANEL_L4
    }
  }
}

}  // namespace dcfr
