// Terminal values of libdcfr: fold and showdown evaluation with exact card
// removal, bit-identical to the reference's evaluators
// (AhanDatta/Poker-Trainer crates/solver/src/eval.rs:40-379).
//
// Layout: one warp works on up to 32 terminals, one per lane; the terminals
// of a showdown group share one board, so their lanes walk the same
// strength-sorted lists. Each lane keeps the reference's sequential
// accumulators — the running opponent sum S (f64, a register) and the 52
// per-card blocker sums (f64, shared memory [53][32], one column per lane;
// row 52 absorbs padding steps) — and adds every opponent hand in the
// reference's order, so every f64 sum rounds exactly as on the CPU.
//
// A sweep is a program: the merge order of the two strength-sorted lists
// (eval.rs:91-143, 250-328), one 32-bit word per step holding the
// shared-memory offsets of the step's two blocker rows, an emit flag and a
// zero-weight flag. Steps are straight-line code: emit and padding steps
// carry weight 0 (their updates are no-ops) and emits are predicated stores.
// A step's blocker sums are loaded before the previous step's update is
// stored, and a load that aliases that update takes it from registers.
//
// Work per showdown group is split over independent warps: the ascending
// pass (win part), the descending pass (lose part) and, when some terminal
// has a fold next to it, the full ascending pass of the paired fold
// (eval.rs:281-300). The second of the two pass warps to finish combines
// win and lose parts (an atomic counter per group, no waiting).
//
// Memory: each warp first copies its 32 reach rows into a per-warp tile in
// its program's step order, Rp[step][lane], so the sweep reads 32 steps as
// one contiguous 4 KB block (cp.async, 16 bytes per copy) and the tile
// writes are coalesced; results go through O[hand][lane] and are
// transposed back into the value rows.
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.hpp"

namespace dcfr {

namespace {

constexpr int CH = TERM_CHUNK;
constexpr int MI_ROWS = 53;  // 52 cards + the padding steps' row
constexpr uint32_t W_EMIT = 0x80000000u;
constexpr uint32_t W_ZERO = 0x40000000u;

__device__ __forceinline__ uint32_t word(uint32_t c1, uint32_t c2, bool emit) {
  return (c1 * 256u) | ((c2 * 256u) << 15) | (emit ? (W_EMIT | W_ZERO) : 0u);
}
__device__ __forceinline__ uint32_t pad_word() { return (52u * 256u) | ((52u * 256u) << 15) | W_ZERO; }

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Shared memory is addressed with 32-bit shared-window addresses and
// explicit ld.shared / st.shared, so these accesses are never generic and
// never ordered against global memory.
__device__ __forceinline__ double lds(uint32_t base, uint32_t off) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(base + off));
  return v;
}
__device__ __forceinline__ void sts(uint32_t base, uint32_t off, double v) {
  asm volatile("st.shared.f64 [%0], %1;" ::"r"(base + off), "d"(v));
}
__device__ __forceinline__ float ldsf(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
__device__ __forceinline__ void stsf(uint32_t addr, float v) { asm volatile("st.shared.f32 [%0], %1;" ::"r"(addr), "f"(v)); }

struct WarpMem {
  uint32_t mi;    // this lane's blocker column: &mi[0][lane]
  uint32_t tile;  // [2][CH][32] f32 staged reach of a chunk of steps
  uint32_t tr;    // [32][33] f32 transpose tile
  int lane;
};

__device__ __forceinline__ void zero_rows(uint32_t mi) {
#pragma unroll 4
  for (int c = 0; c < MI_ROWS; c++) sts(mi, c * 256, 0.0);
}

__device__ __forceinline__ void cp_async16s(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src));
}

// Stages chunk c of Rp (32 steps x 32 lanes, 4 KB) into tile buffer buf:
// lane l copies step row l.
__device__ __forceinline__ void stage(const WarpMem& M, const float* Rp, int c, int buf) {
  const float* src = Rp + ((size_t)c * CH + M.lane) * 32;
  const uint32_t dst = M.tile + (uint32_t)(buf * CH * 32 + M.lane * 32) * 4u;
#pragma unroll
  for (int q = 0; q < 8; q++) cp_async16s(dst + q * 16, src + q * 4);
}

// Runs a program of ns steps (a multiple of CH) over the reach in Rp.
// emit(S, va, vb) is called (predicated) for emit steps with the blocker
// sums of the step's two cards, in program order.
template <class Emit>
__device__ __forceinline__ void sweep(const WarpMem& M, const uint32_t* prog, int ns, const float* Rp, double& S,
                                      Emit emit) {
  if (ns <= 0) return;
  const int lane = M.lane;
  const uint32_t mi = M.mi;
  const int nchunks = ns / CH;
  uint32_t cur = prog[lane];
  uint32_t nxt = nchunks > 1 ? prog[CH + lane] : pad_word();
  stage(M, Rp, 0, 0);
  cp_commit();
  uint32_t pa = 52u * 256u, pb = 52u * 256u;
  double pva = lds(mi, pa), pvb = pva;
  for (int c = 0; c < nchunks; c++) {
    if (c + 1 < nchunks) stage(M, Rp, c + 1, (c + 1) & 1);
    cp_commit();
    cp_wait1();
    __syncwarp();
    const uint32_t t = M.tile + (uint32_t)((c & 1) * CH * 32 + lane) * 4u;
    const uint32_t nxt2 = c + 2 < nchunks ? prog[(c + 2) * CH + lane] : pad_word();
#pragma unroll
    for (int k = 0; k < CH; k++) {
      const uint32_t w = __shfl_sync(0xffffffffu, cur, k);
      const uint32_t oa = w & 0x7FFFu, ob = (w >> 15) & 0x7FFFu;
      const float xf = ldsf(t + k * 128);
      const double x = (w & W_ZERO) ? 0.0 : (double)xf;
      double va = lds(mi, oa), vb = lds(mi, ob);
      va = oa == pa ? pva : (oa == pb ? pvb : va);
      vb = ob == pa ? pva : (ob == pb ? pvb : vb);
      sts(mi, pa, pva);
      sts(mi, pb, pvb);
      if (w & W_EMIT) emit(S, va, vb);
      S += x;
      pva = va + x;
      pvb = vb + x;
      pa = oa;
      pb = ob;
    }
    __syncwarp();
    cur = nxt;
    nxt = nxt2;
  }
  cp_wait0();
  sts(mi, pa, pva);
  sts(mi, pb, pvb);
}

// Rp[pos(h)][lane] = reach of lane's terminal at opponent hand h (0 for
// lanes without a live terminal), pos = posmap[h] (identity when posmap is
// null; NONE32 skips the hand); the zero row gets 0. Through a 32x33
// shared-memory transpose, so row reads and tile writes are coalesced.
__device__ __forceinline__ void fill_rp(const WarpMem& M, const float* reach, int stride, uint32_t slot, bool live, int n,
                        const uint32_t* posmap, float* Rp, int zero_row) {
  const int lane = M.lane;
  const unsigned lm = __ballot_sync(0xffffffffu, live);
  for (int h0 = 0; h0 < n; h0 += 32) {
    float v[32];
#pragma unroll
    for (int t = 0; t < 32; t++) {
      const uint32_t st = __shfl_sync(0xffffffffu, slot, t);
      v[t] = (((lm >> t) & 1) && h0 + lane < n) ? reach[(size_t)st * stride + h0 + lane] : 0.0f;
    }
#pragma unroll
    for (int t = 0; t < 32; t++) stsf(M.tr + (uint32_t)(t * 33 + lane) * 4u, v[t]);  // tr[terminal][hand]
    __syncwarp();
    const uint32_t mypos = h0 + lane < n ? (posmap ? __ldg(posmap + h0 + lane) : (uint32_t)(h0 + lane)) : NONE32;
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const uint32_t pos = __shfl_sync(0xffffffffu, mypos, k);
      const float x = ldsf(M.tr + (uint32_t)(lane * 33 + k) * 4u);
      if (pos != NONE32) Rp[(size_t)pos * 32 + lane] = x;
    }
    __syncwarp();
  }
  Rp[(size_t)zero_row * 32 + lane] = 0.0f;
}

// Value rows of lanes with `write` set: row[h] = O[h][lane] for h < hp.
__device__ __forceinline__ void store_rows(const WarpMem& M, const float* O, float* vals, int stride, uint32_t row, bool write,
                           int hp) {
  const int lane = M.lane;
  const unsigned lm = __ballot_sync(0xffffffffu, write);
  if (!lm) return;
  __syncwarp();
  for (int h0 = 0; h0 < hp; h0 += 32) {
    float v[32];
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = (h0 + k < hp) ? O[(size_t)(h0 + k) * 32 + lane] : 0.0f;
#pragma unroll
    for (int k = 0; k < 32; k++) stsf(M.tr + (uint32_t)(k * 33 + lane) * 4u, v[k]);
    __syncwarp();
#pragma unroll 8
    for (int t = 0; t < 32; t++) {
      const uint32_t r = __shfl_sync(0xffffffffu, row, t);
      const float x = ldsf(M.tr + (uint32_t)(lane * 33 + t) * 4u);
      if (((lm >> t) & 1) && h0 + lane < hp) vals[(size_t)r * stride + h0 + lane] = x;
    }
    __syncwarp();
  }
}

// Fold values from the final sums, in hand order, into O: eval_fold
// (eval.rs:55-63), fold_batch (eval.rs:197-205) and the paired fold of
// showdown_batch (eval.rs:292-300) — `scalar` selects eval_fold's rounding
// and its zero-total rule. The identical opponent hand's reach comes from
// Rp through posmap (identity when null).
__device__ __forceinline__ void fold_emit(const TermArgs& A, const WarpMem& M, const float* Rp, const uint32_t* posmap, int zero_row,
                          float* O, double total, double pay, bool scalar) {
  const int p = A.p, lane = M.lane;
  const int np = A.n[p], hp = A.hp[p];
  const uint2* er = A.emit_rec[p];
  for (int h0 = 0; h0 < hp; h0 += 32) {
    const uint2 rec = h0 + lane < np ? __ldg(er + h0 + lane) : make_uint2(52u * 256u | ((52u * 256u) << 15), NONE32);
    float sw[32];
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const uint32_t sm = __shfl_sync(0xffffffffu, rec.y, k);
      uint32_t pos = (uint32_t)zero_row;
      if (sm != NONE32) {
        const uint32_t q = posmap ? __ldg(posmap + sm) : sm;
        pos = q == NONE32 ? (uint32_t)zero_row : q;
      }
      sw[k] = Rp[(size_t)pos * 32 + lane];
    }
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const uint32_t w = __shfl_sync(0xffffffffu, rec.x, k);
      const int h = h0 + k;
      float f = 0.0f;
      if (h < np) {
        const double a = lds(M.mi, w & 0x7FFFu), b = lds(M.mi, (w >> 15) & 0x7FFFu);
        const double s = (double)sw[k];
        if (scalar)
          f = total == 0.0 ? 0.0f : (float)(pay * ((total - (a + b)) + s));
        else
          f = (float)(pay * (((total - a) - b) + s));
      }
      if (h < hp) O[(size_t)h * 32 + lane] = f;
    }
  }
}

__device__ __forceinline__ EntryD ld_entry(const EntryD* e) {
  uint2 v = __ldg(reinterpret_cast<const uint2*>(e));
  EntryD r;
  r.strength = v.x;
  r.idx = (uint16_t)(v.y & 0xFFFFu);
  r.c1 = (uint8_t)((v.y >> 16) & 0xFFu);
  r.c2 = (uint8_t)(v.y >> 24);
  return r;
}

// add_ties (eval.rs:347-379) into O, only for lanes whose tie payoff is
// nonzero (mid-street roots, rake). Sequential, in the reference's order,
// reading the reach rows directly.
__device__ void add_ties(const TermArgs& A, const WarpMem& M, const float* rr, bool live, const EntryD* mine,
                         const EntryD* theirs, int cm, int ct, double tie, bool write, float* O) {
  const uint32_t mi = M.mi;
  zero_rows(mi);
  int k = 0, j = 0;
  while (k < cm) {
    const uint32_t s = ld_entry(mine + k).strength;
    while (j < ct && ld_entry(theirs + j).strength < s) j++;
    double eq_sum = 0.0;
    int jj = j;
    while (jj < ct) {
      EntryD e = ld_entry(theirs + jj);
      if (e.strength != s) break;
      double w = live ? (double)rr[e.idx] : 0.0;
      eq_sum += w;
      sts(mi, e.c1 * 256u, lds(mi, e.c1 * 256u) + w);
      sts(mi, e.c2 * 256u, lds(mi, e.c2 * 256u) + w);
      jj++;
    }
    while (k < cm) {
      EntryD e = ld_entry(mine + k);
      if (e.strength != s) break;
      uint32_t sm = __ldg(A.same[A.p] + e.idx);
      double sw = (sm != NONE32 && live) ? (double)rr[sm] : 0.0;
      double eq = (eq_sum - (lds(mi, e.c1 * 256u) + lds(mi, e.c2 * 256u))) + sw;
      if (write) O[(size_t)e.idx * 32 + M.lane] += (float)(tie * eq);
      k++;
    }
    for (int q = j; q < jj; q++) {
      EntryD e = ld_entry(theirs + q);
      sts(mi, e.c1 * 256u, 0.0);
      sts(mi, e.c2 * 256u, 0.0);
    }
  }
}

}  // namespace

// Shared memory per warp: blocker rows, two staging tiles, a transpose tile.
constexpr size_t TERM_WARP_BYTES = MI_ROWS * 32 * 8 + 2 * CH * 32 * 4 + 32 * 33 * 4;

__global__ void __launch_bounds__(TERM_WARPS * 32) terminal_kernel(TermArgs A, const TermGroup* __restrict__ groups,
                                                                    const TermLane* __restrict__ lanes,
                                                                    const TermTask* __restrict__ tasks, int ntasks) {
  extern __shared__ unsigned char smem_term[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tid = blockIdx.x * TERM_WARPS + warp;
  if (tid >= ntasks) return;
  const uint32_t wbase = (uint32_t)__cvta_generic_to_shared(smem_term) + (uint32_t)(warp * TERM_WARP_BYTES);
  WarpMem M;
  M.mi = wbase + lane * 8;
  M.tile = wbase + MI_ROWS * 256;
  M.tr = M.tile + 2 * CH * 32 * 4;
  M.lane = lane;
  // Per-warp scratch: Rp [pstride+1][32] and O [stride][32] (f32).
  float* Rp = A.warp_scratch + (size_t)tid * A.warp_scratch_floats;
  float* O = Rp + (size_t)(A.pstride + 1) * 32;
  const int zero_row = A.pstride;
  const TermTask task = tasks[tid];
  const TermGroup G = groups[task.group];
  const int p = A.p, o = p ^ 1;
  const bool act = lane < (int)G.count;
  TermLane T;
  if (act) {
    T = lanes[G.first + lane];
  } else {
    T.slot = 0;
    T.row = 0;
    T.frow = NONE32;
    T.pad = 0;
    T.a = T.b = T.c = T.d = 0.0;
  }
  const bool live = act && A.alive[T.slot] != 0;
  const int hp = A.hp[p];

  if (task.role == R_FOLD) {
    // Opponent sums in hand order, then every hand's fold value.
    fill_rp(M, A.reach, A.stride, T.slot, live, A.n[o], nullptr, Rp, zero_row);
    zero_rows(M.mi);
    __syncwarp();
    double S = 0.0;
    sweep(M, A.fold_prog[o], (A.n[o] + CH - 1) / CH * CH, Rp, S, [](double, double, double) {});
    fold_emit(A, M, Rp, nullptr, zero_row, O, S, T.a, G.kind == T_FOLD_SCALAR);
    store_rows(M, O, A.vals, A.stride, T.row, live, hp);
    return;
  }

  const size_t bp = (size_t)G.board * 2 + p;
  const int dir = task.role == R_ASC ? 0 : task.role == R_DESC ? 1 : 2;
  const size_t pi = bp * 3 + dir;
  const uint32_t* prog = A.progs + pi * A.pstride;
  const int ns = (int)A.prog_count[pi];
  const uint32_t* posmap = A.posmap + pi * A.tstride;
  fill_rp(M, A.reach, A.stride, T.slot, live, A.n[o], posmap, Rp, zero_row);
  zero_rows(M.mi);
  __syncwarp();
  double S = 0.0;

  if (task.role == R_PAIRED) {
    // All opponent hands in strength order, then the fold read off the sums.
    const bool has_fold = live && T.frow != NONE32;
    sweep(M, prog, ns, Rp, S, [](double, double, double) {});
    fold_emit(A, M, Rp, posmap, zero_row, O, S, T.d, false);
    store_rows(M, O, A.vals, A.stride, T.frow, has_fold, hp);
    return;
  }

  const bool batch = G.kind == T_SHOWDOWN_BATCH;
  const int cm = (int)A.table_count[bp];
  double* W = A.group_scratch + (size_t)task.wgroup * 2 * A.nmax * 32;
  double* L = W + (size_t)A.nmax * 32;
  if (task.role == R_ASC) {
    // Win part (eval.rs:271 batched, eval.rs:112 scalar), entries ascending.
    const double win = T.a;
    int i = 0;
    sweep(M, prog, ns, Rp, S, [&](double Sv, double va, double vb) {
      W[(size_t)i * 32 + lane] = batch ? win * ((Sv - va) - vb) : win * (Sv - (va + vb));
      i++;
    });
  } else {
    // Lose part (eval.rs:324 batched, eval.rs:139 scalar), entries descending.
    const double lose = T.b;
    int i = cm - 1;
    sweep(M, prog, ns, Rp, S, [&](double Sv, double va, double vb) {
      L[(size_t)i * 32 + lane] = batch ? lose * ((Sv - va) - vb) : lose * (Sv - (va + vb));
      i--;
    });
  }
  // The second of the two pass warps combines: out = win + lose, one f64
  // rounding (batched, eval.rs:324-333) or two f32 values added (scalar,
  // eval.rs:112, 139).
  __threadfence();
  __syncwarp();
  uint32_t prev = 0;
  if (lane == 0) prev = atomicAdd(A.counters + task.wgroup, 1u);
  prev = __shfl_sync(0xffffffffu, prev, 0);
  if (prev != 1) return;
  __threadfence();
  const EntryD* mine = A.tables + bp * A.tstride;
  for (int h = 0; h < hp; h++) O[(size_t)h * 32 + lane] = 0.0f;
  for (int i0 = 0; i0 < cm; i0 += 16) {
    double Wv[16], Lv[16];
    uint32_t dst[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
      const int i = i0 + k;
      if (i < cm) {
        Wv[k] = __ldcg(W + (size_t)i * 32 + lane);
        Lv[k] = __ldcg(L + (size_t)i * 32 + lane);
        dst[k] = ld_entry(mine + i).idx;
      }
    }
#pragma unroll
    for (int k = 0; k < 16; k++)
      if (i0 + k < cm) O[(size_t)dst[k] * 32 + lane] = batch ? (float)(Wv[k] + Lv[k]) : (float)Wv[k] + (float)Lv[k];
  }
  const bool tie = live && T.c != 0.0;
  if (__any_sync(0xffffffffu, tie)) {
    const EntryD* theirs = A.tables + ((size_t)G.board * 2 + o) * A.tstride;
    const int ct = (int)A.table_count[(size_t)G.board * 2 + o];
    add_ties(A, M, A.reach + (size_t)T.slot * A.stride, live, mine, theirs, cm, ct, T.c, tie, O);
  }
  store_rows(M, O, A.vals, A.stride, T.row, live, hp);
  if (lane == 0) A.counters[task.wgroup] = 0u;
}

// Programs of one board and traverser (one thread per board, player and
// direction): ascending (eval.rs:91-116) and descending (eval.rs:118-143)
// merges of the traverser's and the opponent's strength-sorted lists, and
// the opponent list alone in strength order (the paired fold,
// eval.rs:281-291); posmap maps an opponent hand to its step.
__global__ void program_kernel(const EntryD* __restrict__ tables, const uint32_t* __restrict__ count, int tstride,
                               uint32_t* progs, uint32_t* prog_count, uint32_t* posmap, int pstride, int nprog) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= nprog) return;
  const int dir = id % 3, bp = id / 3, b = bp >> 1, p = bp & 1, o = p ^ 1;
  const EntryD* mine = tables + (size_t)bp * tstride;
  const EntryD* theirs = tables + ((size_t)b * 2 + o) * tstride;
  const int cm = (int)count[bp], ct = (int)count[(size_t)b * 2 + o];
  uint32_t* out = progs + (size_t)id * pstride;
  uint32_t* pos = posmap + (size_t)id * tstride;
  for (int h = 0; h < tstride; h++) pos[h] = NONE32;
  int k = 0;
  auto acc = [&](const EntryD& e) {
    pos[e.idx] = (uint32_t)k;
    out[k++] = word(e.c1, e.c2, false);
  };
  if (dir == 0) {
    int i = 0, j = 0;
    while (i < cm) {
      const uint32_t s = mine[i].strength;
      while (j < ct && theirs[j].strength < s) acc(theirs[j++]);
      while (i < cm && mine[i].strength == s) {
        out[k++] = word(mine[i].c1, mine[i].c2, true);
        i++;
      }
    }
  } else if (dir == 1) {
    int i = cm, j = ct;
    while (i > 0) {
      const uint32_t s = mine[i - 1].strength;
      while (j > 0 && theirs[j - 1].strength > s) acc(theirs[--j]);
      while (i > 0 && mine[i - 1].strength == s) {
        out[k++] = word(mine[i - 1].c1, mine[i - 1].c2, true);
        i--;
      }
    }
  } else {
    for (int j = 0; j < ct; j++) acc(theirs[j]);
  }
  // Pad to whole chunks: weight-0 steps on the spare row 52.
  while (k % CH) out[k++] = pad_word();
  prog_count[id] = (uint32_t)k;
}

// Per player: hands in hand order as accumulate steps (fold sums, padded
// to whole chunks) and per-hand emit records (blocker rows, identical
// opponent hand).
__global__ void hand_program_kernel(const uint8_t* c1, const uint8_t* c2, const uint32_t* same, int n, int npad,
                                    uint32_t* fold_prog, uint2* emit_rec) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < npad) fold_prog[i] = i < n ? word(c1[i], c2[i], false) : pad_word();
  if (i < n) emit_rec[i] = make_uint2(word(c1[i], c2[i], false), same[i]);
}

size_t terminal_smem_bytes() { return (size_t)TERM_WARPS * TERM_WARP_BYTES; }

cudaError_t terminal_kernel_setup() {
  return cudaFuncSetAttribute(terminal_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)terminal_smem_bytes());
}

void launch_terminal(const TermArgs& A, const TermGroup* groups, const TermLane* lanes, const TermTask* tasks,
                     int ntasks, cudaStream_t s) {
  if (ntasks <= 0) return;
  const int blocks = (ntasks + TERM_WARPS - 1) / TERM_WARPS;
  terminal_kernel<<<blocks, TERM_WARPS * 32, terminal_smem_bytes(), s>>>(A, groups, lanes, tasks, ntasks);
}

void launch_programs(const EntryD* tables, const uint32_t* count, int tstride, uint32_t* progs, uint32_t* prog_count,
                     uint32_t* posmap, int pstride, int nboards, cudaStream_t s) {
  const int nprog = nboards * 2 * 3;
  program_kernel<<<(nprog + 63) / 64, 64, 0, s>>>(tables, count, tstride, progs, prog_count, posmap, pstride, nprog);
}

void launch_hand_program(const uint8_t* c1, const uint8_t* c2, const uint32_t* same, int n, int npad,
                         uint32_t* fold_prog, uint2* emit_rec, cudaStream_t s) {
  if (npad > 0) hand_program_kernel<<<(npad + 255) / 256, 256, 0, s>>>(c1, c2, same, n, npad, fold_prog, emit_rec);
}

}  // namespace dcfr
