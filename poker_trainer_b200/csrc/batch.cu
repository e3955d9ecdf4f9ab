// Batched river solves: hundreds of independent river subgames of uneven tree
// size solved together by one persistent kernel per block of iterations,
// launched from a captured CUDA graph.
//
// Every spot is a complete river game (its own board, ranges, pot, stacks
// and bet menu) built by the same host code as a single solve (game.cpp), so
// its tree, storage order and arithmetic are those of the reference solver
// (crates/solver/src/tree.rs, cfr.rs, river.rs, eval.rs). The device work of
// one spot is the work of the single-solve kernels, done by one block:
//   * down: opponent nodes in breadth-first order with a block barrier at
//     each new depth (down_item, row_items.cuh);
//   * terminals: one warp per terminal over the spot's staged scan layout
//     (warp_terminal_task, warp_terminal.cuh), showdowns then folds;
//   * up: deepest level first (up_item); a thread keeps the same 4 hands
//     throughout, so no barrier is needed between up nodes.
// Liveness flags (the dead-subtree rule, cfr.rs:267-274) and the current
// discounts live in the block's shared memory. Blocks take spots from a
// work counter, longest spots first, and run `iters` iterations of a spot
// before taking the next, so one launch needs no grid-wide barrier.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

#include "batch.hpp"
#include "row_items.cuh"
#include "warp_terminal.cuh"

namespace dcfr {

namespace {

struct SpotD {
  uint64_t store;  // float offset of the spot's storage block (regrets and sums)
  uint64_t vals;   // float offset of its value rows (nodes x stride)
  uint64_t reach;  // float offset of its reach rows (slots x stride)
  uint32_t hands;  // offset of its hand cards: player q at hands + q * stride
  uint32_t same;   // offset of its identical-hand maps: player q at same + q * stride
  uint32_t root;   // offset of its root rows [2][stride] (opponent weights per traverser)
  uint32_t layout; // showdown layout; the fold layout is layout + 1
  uint32_t down_first[2], down_count[2];
  uint32_t up_first[2], up_count[2];
  uint32_t term_first[2], term_sd[2], term_count[2];
  int32_t n[2], hp[2], stride, slots;
};

struct BatchArgs {
  float* regrets;
  float* sums;
  float* reach;
  float* vals;
  float* root_out;  // best-response / average root rows, same layout as roots
  const uint8_t* hc1;
  const uint8_t* hc2;
  const uint32_t* same;
  const float* roots;
  const uint16_t* cat;
  const uint16_t* seg;
  const uint4* rec;
  const DownTask* down;
  const UpTask* up;
  const FastTask* term;
  const SpotD* spots;
  const uint32_t* order;
  int nspots;
  const DiscountD* disc_table;
  uint32_t disc_len;
  const uint32_t* counter;  // iterations done before this launch
  uint32_t* work;           // spots taken in this launch
  int cstride, tstride;
  int max_slots, max_stride;
  int iters;
};

struct BatchSmem {
  size_t alive, disc, work, same, cat, rec, seg, warp0, row_bytes, warp_bytes, total;
  __host__ __device__ BatchSmem(int max_slots, int max_stride, int cstride, int tstride, int warps) {
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    alive = 0;
    disc = up16(alive + (size_t)max_slots * 4);
    work = up16(disc + sizeof(DiscountD));
    same = up16(work + 16);
    cat = up16(same + (size_t)max_stride * 2);
    rec = up16(cat + (size_t)cstride * 2);
    seg = up16(rec + (size_t)tstride * 16);
    warp0 = up16(seg + FAST_SEGS * 2);
    row_bytes = up16((size_t)max_stride * 4);
    warp_bytes = row_bytes + up16(warp_prefix_entries(cstride) * 8);
    total = warp0 + (size_t)warps * warp_bytes;
  }
};

template <int MODE, int MAXA>
__global__ void __launch_bounds__(BATCH_MAX_THREADS) batch_kernel(BatchArgs B) {
  extern __shared__ __align__(16) unsigned char smem_b[];
  const int NT = (int)blockDim.x, W = NT >> 5;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const BatchSmem L_(B.max_slots, B.max_stride, B.cstride, B.tstride, W);
  uint32_t* alive = reinterpret_cast<uint32_t*>(smem_b + L_.alive);
  DiscountD* disc = reinterpret_cast<DiscountD*>(smem_b + L_.disc);
  int* s_work = reinterpret_cast<int*>(smem_b + L_.work);
  uint16_t* ssame = reinterpret_cast<uint16_t*>(smem_b + L_.same);
  uint16_t* scat = reinterpret_cast<uint16_t*>(smem_b + L_.cat);
  uint4* srec = reinterpret_cast<uint4*>(smem_b + L_.rec);
  uint16_t* sseg = reinterpret_cast<uint16_t*>(smem_b + L_.seg);
  float* wrow = reinterpret_cast<float*>(smem_b + L_.warp0 + (size_t)warp * L_.warp_bytes);
  long long* G = reinterpret_cast<long long*>(smem_b + L_.warp0 + (size_t)warp * L_.warp_bytes + L_.row_bytes);
  const uint32_t t0 = *B.counter;

  for (;;) {
    __syncthreads();  // the previous spot is finished with shared memory
    if (tid == 0) *s_work = (int)atomicAdd(B.work, 1u);
    __syncthreads();
    const int w = *s_work;
    if (w >= B.nspots) break;
    const SpotD S = B.spots[B.order[w]];
    RowArgs A;
    A.regrets = B.regrets + S.store;
    A.sums = B.sums + S.store;
    A.reach = B.reach + S.reach;
    A.vals = B.vals + S.vals;
    A.alive = alive;
    for (int q = 0; q < 2; q++) {
      A.hc1[q] = B.hc1 + S.hands + (size_t)q * S.stride;
      A.hc2[q] = B.hc2 + S.hands + (size_t)q * S.stride;
      A.n[q] = S.n[q];
      A.hp[q] = S.hp[q];
    }
    A.perm = nullptr;
    A.chance_cards = nullptr;
    A.iso = nullptr;
    A.disc = disc;
    A.stride = S.stride;
    const int iters = MODE == M_CFR ? B.iters : 1;
    for (int it = 0; it < iters; it++) {
      if (MODE == M_CFR && tid == 0) {
        const uint32_t t = t0 + 1u + (uint32_t)it;
        *disc = B.disc_table[t < B.disc_len ? t : B.disc_len - 1];
      }
      for (int p = 0; p < 2; p++) {
        const int o = p ^ 1;
        A.p = p;
        for (int i = tid; i < S.slots; i += NT) alive[i] = 0u;
        for (int h = tid; h < S.hp[p]; h += NT) {
          const uint32_t sm = h < S.n[p] ? B.same[S.same + (size_t)p * S.stride + h] : NONE32;
          ssame[h] = sm == NONE32 ? (uint16_t)0xFFFF : (uint16_t)sm;
        }
        const float* root = B.roots + S.root + (size_t)p * S.stride;
        for (int i = tid; i < S.stride / 4; i += NT) st4(A.reach + 4 * i, ld4(root + 4 * i));
        __syncthreads();
        if (tid == 0) alive[0] = 1u;
        __syncthreads();
        // Down: opponent splits, breadth first.
        const int dpass = (S.hp[o] + NT * VEC - 1) / (NT * VEC);
        for (uint32_t i = 0; i < S.down_count[p]; i++) {
          const DownTask T = B.down[S.down_first[p] + i];
          if (T.kind & LEVEL_BREAK) __syncthreads();
          for (int ps = 0; ps < dpass; ps++) down_item<MODE, MAXA, D_OPP_SPLIT>(A, T, (ps * NT + tid) * VEC, lane);
        }
        __syncthreads();
        // Terminals: showdowns on the board's layout, then folds.
        FastArgs F;
        F.reach = A.reach;
        F.vals = A.vals;
        F.alive = alive;
        F.n[0] = S.n[0];
        F.n[1] = S.n[1];
        F.hp[0] = S.hp[0];
        F.hp[1] = S.hp[1];
        F.stride = S.stride;
        F.p = p;
        for (int gsel = 0; gsel < 2; gsel++) {
          const uint32_t first = S.term_first[p] + (gsel ? S.term_sd[p] : 0u);
          const uint32_t count = gsel ? S.term_count[p] - S.term_sd[p] : S.term_sd[p];
          if (count == 0) continue;
          const size_t lay = (size_t)(S.layout + gsel) * 2 + p;
          const uint16_t* gseg = B.seg + lay * FAST_SEGS;
          if (tid < FAST_SEGS) sseg[tid] = gseg[tid];
          const int L = gseg[FAST_SEGS - 1];
          const uint16_t* gcat = B.cat + lay * B.cstride;
          for (int k = tid; k < L; k += NT) scat[k] = gcat[k];
          const uint4* grec = B.rec + lay * B.tstride;
          for (int h = tid; h < S.n[p]; h += NT) srec[h] = grec[h];
          __syncthreads();
          const WarpLayout Y{ssame, scat, srec, sseg, L};
          for (uint32_t ti = warp; ti < count; ti += W) {
            const FastTask T = B.term[first + ti];
            if (alive[T.slot] == 0) continue;
            warp_terminal_task<float>(F, T, Y, wrow, G, lane);
          }
          __syncthreads();
        }
        // Up: deepest first; each thread owns the same hands as in the down pass.
        const int upass = (S.hp[p] + NT * VEC - 1) / (NT * VEC);
        for (uint32_t i = 0; i < S.up_count[p]; i++) {
          const UpTask T = B.up[S.up_first[p] + i];
          for (int ps = 0; ps < upass; ps++) {
            const int h0 = (ps * NT + tid) * VEC;
            if ((T.kind & KIND_MASK) == U_OWN) up_item<MODE, MAXA, U_OWN>(A, T, h0);
            else up_item<MODE, MAXA, U_OPP_SUM>(A, T, h0);
          }
        }
        __syncthreads();
        if (MODE != M_CFR) {
          float* dst = B.root_out + S.root + (size_t)p * S.stride;
          for (int i = tid; i < S.stride / 4; i += NT) st4(dst + 4 * i, ld4(A.vals + 4 * i));
          __syncthreads();
        }
      }
    }
  }
}

__global__ void batch_advance_kernel(uint32_t* counter, uint32_t n, uint32_t* work) {
  *counter += n;
  *work = 0u;
}

template <int MODE>
const void* kernel_for(int maxa) {
  if (maxa <= 4) return (const void*)batch_kernel<MODE, 4>;
  if (maxa <= 8) return (const void*)batch_kernel<MODE, 8>;
  return (const void*)batch_kernel<MODE, MAX_ACTIONS>;
}

const void* batch_kernel_ptr(int mode, int maxa) {
  if (mode == M_CFR) return kernel_for<M_CFR>(maxa);
  if (mode == M_BR) return kernel_for<M_BR>(maxa);
  return kernel_for<M_AVG>(maxa);
}

Status cuda_st(cudaError_t e, const char* what) { return cuda_status(e, what); }

#define BK(call)                                  \
  do {                                            \
    Status _s = cuda_st((call), #call);           \
    if (!_s.ok()) return _s;                      \
  } while (0)

template <class T>
Status balloc(T*& p, size_t count, const char* what) {
  p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
  if (e != cudaSuccess) {
    Status s = cuda_status(e, what);
    s.msg += " (" + std::to_string(count * sizeof(T)) + " bytes)";
    return s;
  }
  return Status();
}

template <class T>
void bfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <class T>
Status upload(T*& d, const std::vector<T>& h, const char* what) {
  Status s = balloc(d, h.size(), what);
  if (!s.ok()) return s;
  if (!h.empty()) BK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return Status();
}

inline int pad8(int n) { return (n + 7) & ~7; }

}  // namespace

struct Batch::Impl {
  std::vector<Game> games;
  std::vector<SpotD> spots;
  std::vector<std::vector<uint64_t>> node_off;  // per spot, per node: float offset of a player block in the spot
  std::vector<uint64_t> spot_len;               // storage floats per spot
  std::vector<double> cost;
  int maxa = 1, max_slots = 1, max_stride = 8, tstride = 1, cstride = 8;
  uint64_t total_store = 0;
  // Device.
  cudaStream_t stream = nullptr;
  float *regrets = nullptr, *sums = nullptr, *reach = nullptr, *vals = nullptr, *roots = nullptr, *root_out = nullptr;
  uint8_t *hc1 = nullptr, *hc2 = nullptr;
  uint32_t* same = nullptr;
  uint16_t *cat = nullptr, *seg = nullptr;
  uint4* rec = nullptr;
  EntryD* tables = nullptr;
  uint32_t* tcount = nullptr;
  uint8_t* boards = nullptr;
  DownTask* down = nullptr;
  UpTask* up = nullptr;
  FastTask* term = nullptr;
  SpotD* d_spots = nullptr;
  uint32_t *order_lpt = nullptr, *order_nat = nullptr;
  DiscountD* disc = nullptr;
  uint32_t disc_len = 0;
  uint32_t* counter = nullptr;
  uint32_t* work = nullptr;
  uint32_t iterations = 0;
  dcfr_batch_tuning tuning{};
  cudaGraphExec_t graph = nullptr;
  uint32_t graph_iters = 0;
  int sms = 148;
  uint64_t launches = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = 0.0;

  ~Impl();
  Status init(const dcfr_config* cfgs, int count);
  BatchArgs args(int mode, uint32_t iters, bool lpt) const;
  Status launch(int mode, uint32_t iters, const dcfr_batch_tuning& t);
  Status ensure_discounts(uint32_t max_t);
  Status capture(uint32_t iters);
  Status run(uint32_t n);
};

Batch::Impl::~Impl() {
  if (stream) cudaStreamSynchronize(stream);
  if (graph) cudaGraphExecDestroy(graph);
  bfree(regrets);
  bfree(sums);
  bfree(reach);
  bfree(vals);
  bfree(roots);
  bfree(root_out);
  bfree(hc1);
  bfree(hc2);
  bfree(same);
  bfree(cat);
  bfree(seg);
  bfree(rec);
  bfree(tables);
  bfree(tcount);
  bfree(boards);
  bfree(down);
  bfree(up);
  bfree(term);
  bfree(d_spots);
  bfree(order_lpt);
  bfree(order_nat);
  bfree(disc);
  bfree(counter);
  bfree(work);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stream) cudaStreamDestroy(stream);
}

// DcfrParams -> Discount (cfr.rs:86-106); defined in engine.cu.
DiscountD discount_of(uint32_t t, const dcfr_params& prm);

Status Batch::Impl::ensure_discounts(uint32_t max_t) {
  if (disc && max_t < disc_len) return Status();
  const uint32_t len = std::max<uint32_t>(max_t + 1, disc_len * 2);
  std::vector<DiscountD> tab(len);
  for (uint32_t t = 0; t < len; t++) tab[t] = discount_of(t, games[0].cfg.dcfr);
  BK(cudaStreamSynchronize(stream));
  if (graph) {
    cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  bfree(disc);
  Status s = upload(disc, tab, "discounts");
  disc_len = len;
  return s;
}

Status Batch::Impl::init(const dcfr_config* cfgs, int count) {
  Status s;
  BK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  BK(cudaEventCreate(&ev0));
  BK(cudaEventCreate(&ev1));
  int dev = 0;
  BK(cudaGetDevice(&dev));
  BK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  games.resize(count);
  for (int i = 0; i < count; i++) {
    const dcfr_config& c = cfgs[i];
    if (c.board_len != 5 || c.root.street != DCFR_RIVER) {
      s.code = DCFR_ERR_UNSUPPORTED;
      s.msg = "spot " + std::to_string(i) + ": the batched solve takes river spots (5-card board, river root)";
      return s;
    }
    if (c.precision != DCFR_PRECISION_FAST) {
      s.code = DCFR_ERR_UNSUPPORTED;
      s.msg = "spot " + std::to_string(i) + ": the batched solve runs in fast precision";
      return s;
    }
    if (std::memcmp(&c.dcfr, &cfgs[0].dcfr, sizeof c.dcfr) != 0) {
      s.code = DCFR_ERR_INVALID_ARG;
      s.msg = "spot " + std::to_string(i) + ": all spots of a batch share one DcfrParams";
      return s;
    }
    std::string msg;
    int rc = build_game(c, games[i], msg, true);
    if (rc) {
      s.code = rc;
      s.msg = "spot " + std::to_string(i) + ": " + msg;
      return s;
    }
    if (games[i].compressed) {
      s.code = DCFR_ERR_UNSUPPORTED;
      s.msg = "spot " + std::to_string(i) + ": the batched solve runs f32 storage";
      return s;
    }
  }
  // Host plans and the layout of every device array.
  std::vector<DownTask> hdown;
  std::vector<UpTask> hup;
  std::vector<FastTask> hterm;
  std::vector<uint8_t> h1, h2, hb;
  std::vector<uint32_t> hs;
  std::vector<float> hroot;
  uint64_t vals_off = 0, reach_off = 0;
  spots.resize(count);
  node_off.resize(count);
  spot_len.resize(count);
  cost.resize(count);
  for (int i = 0; i < count; i++) tstride = std::max(tstride, std::max(games[i].n[0], games[i].n[1]));
  cstride = (3 * tstride + 7) / 8 * 8;
  for (int i = 0; i < count; i++) {
    const Game& g = games[i];
    SpotD& S = spots[i];
    std::memset(&S, 0, sizeof S);
    const int hp0 = pad8(g.n[0]), hp1 = pad8(g.n[1]), stride = std::max(hp0, hp1);
    S.n[0] = g.n[0];
    S.n[1] = g.n[1];
    S.hp[0] = hp0;
    S.hp[1] = hp1;
    S.stride = stride;
    max_stride = std::max(max_stride, stride);
    const size_t N = g.nodes.size();
    // Storage: player blocks [a][hp_q] in the reference's node order.
    const std::vector<uint32_t> players = players_in_storage_order(g);
    node_off[i].assign(N, 0);
    uint64_t len = 0;
    for (uint32_t v : players) {
      node_off[i][v] = len;
      len += (uint64_t)g.nodes[v].nchild * (uint64_t)(g.nodes[v].player ? hp1 : hp0);
      maxa = std::max<int>(maxa, g.nodes[v].nchild);
    }
    S.store = total_store;
    spot_len[i] = len;
    total_store += len;
    // Hands, identical-hand maps, root rows, board.
    S.hands = (uint32_t)h1.size();
    S.same = (uint32_t)hs.size();
    S.root = (uint32_t)hroot.size();
    for (int q = 0; q < 2; q++) {
      const int hq = q ? hp1 : hp0;
      for (int h = 0; h < stride; h++) {
        const bool in = h < g.n[q];
        h1.push_back(in ? g.c1[q][h] : 255);
        h2.push_back(in ? g.c2[q][h] : 255);
        hs.push_back(in ? g.same[q][h] : NONE32);
      }
      (void)hq;
    }
    for (int p = 0; p < 2; p++)
      for (int h = 0; h < stride; h++) hroot.push_back(h < g.n[p ^ 1] ? g.weights[p ^ 1][h] : 0.0f);
    for (int k = 0; k < 5; k++) hb.push_back((uint8_t)g.board[k]);
    S.layout = (uint32_t)(2 * i);
    // Traversal plans: slots, down tasks (BFS, level breaks), up tasks
    // (deepest first), terminals (showdowns with paired folds, then folds).
    int slots_max = 1;
    uint64_t work_units = 0;
    for (int p = 0; p < 2; p++) {
      const int o = p ^ 1;
      std::vector<uint32_t> slot(N, 0), depth(N, 0);
      std::vector<std::pair<uint32_t, UpTask>> ups;
      std::vector<FastTask> sds, folds;
      uint32_t next_slot = 1;
      std::vector<uint32_t> queue{0};
      uint32_t prev_depth = 0;
      S.down_first[p] = (uint32_t)hdown.size();
      for (size_t qi = 0; qi < queue.size(); qi++) {
        const uint32_t v = queue[qi];
        const GNode& nd = g.nodes[v];
        const uint32_t sv = slot[v];
        if (nd.kind == N_PLAYER) {
          const bool own = nd.player == p;
          const uint32_t first_slot = own ? sv : next_slot;
          if (!own) next_slot += nd.nchild;
          for (uint32_t c = 0; c < nd.nchild; c++) {
            slot[nd.first + c] = own ? sv : first_slot + c;
            depth[nd.first + c] = depth[v] + 1;
            queue.push_back(nd.first + c);
          }
          if (!own) {
            DownTask t{D_OPP_SPLIT, sv, first_slot, nd.nchild, node_off[i][v], 0, 0.0f};
            if (hdown.size() > S.down_first[p] && depth[v] != prev_depth) t.kind |= LEVEL_BREAK;
            prev_depth = depth[v];
            hdown.push_back(t);
          }
          ups.push_back({depth[v], UpTask{own ? (uint32_t)U_OWN : (uint32_t)U_OPP_SUM, sv, v, nd.first, nd.nchild,
                                          first_slot, node_off[i][v], 0, 0, 0, 0}});
          work_units += nd.nchild;
        } else if (nd.kind == N_FOLD || nd.kind == N_SHOWDOWN) {
          // Every terminal of a river spot sits below a river decision node:
          // batched evaluation (cfr.rs:282-284, river.rs:163-249), with a fold
          // beside a showdown under the traverser's own decision read off the
          // showdown's sums.
          const GNode& par = g.nodes[nd.parent];
          const double hpot = g.half_pot, norm = g.norm;
          if (nd.kind == N_FOLD) {
            bool paired = false;
            if (par.player == p)
              for (uint32_t c = par.first; c < par.first + par.nchild; c++)
                if (g.nodes[c].kind == N_SHOWDOWN) paired = true;
            if (paired) continue;
            const int f = nd.player;
            const double val = f == p ? -(hpot + (double)nd.invest[p]) : hpot + (double)nd.invest[f] - (double)nd.rake;
            folds.push_back(FastTask{T_FOLD_BATCH, 1, sv, v, NONE32, {0, 0, 0}, val * norm, 0.0, 0.0, 0.0});
          } else {
            const double rake = (double)nd.rake;
            FastTask t{T_SHOWDOWN_BATCH, 0, sv, v, NONE32, {0, 0, 0},
                       (hpot + (double)nd.invest[o] - rake) * norm, -(hpot + (double)nd.invest[p]) * norm,
                       0.5 * ((double)(nd.invest[o] - nd.invest[p]) - rake) * norm, 0.0};
            if (par.player == p)
              for (uint32_t c = par.first; c < par.first + par.nchild; c++)
                if (g.nodes[c].kind == N_FOLD) {
                  const GNode& fn = g.nodes[c];
                  const int f = fn.player;
                  const double val =
                      f == p ? -(hpot + (double)fn.invest[p]) : hpot + (double)fn.invest[f] - (double)fn.rake;
                  t.frow = c;
                  t.d = val * norm;
                }
            sds.push_back(t);
          }
        }
      }
      S.down_count[p] = (uint32_t)(hdown.size() - S.down_first[p]);
      std::stable_sort(ups.begin(), ups.end(),
                       [](const std::pair<uint32_t, UpTask>& a, const std::pair<uint32_t, UpTask>& b) {
                         return a.first > b.first;
                       });
      S.up_first[p] = (uint32_t)hup.size();
      for (auto& x : ups) hup.push_back(x.second);
      S.up_count[p] = (uint32_t)ups.size();
      S.term_first[p] = (uint32_t)hterm.size();
      hterm.insert(hterm.end(), sds.begin(), sds.end());
      hterm.insert(hterm.end(), folds.begin(), folds.end());
      S.term_sd[p] = (uint32_t)sds.size();
      S.term_count[p] = (uint32_t)(sds.size() + folds.size());
      slots_max = std::max<int>(slots_max, (int)next_slot);
      work_units += sds.size() * 3 + folds.size();
    }
    S.slots = slots_max;
    max_slots = std::max(max_slots, slots_max);
    S.vals = vals_off;
    vals_off += (uint64_t)N * stride;
    S.reach = reach_off;
    reach_off += (uint64_t)slots_max * stride;
    cost[i] = (double)work_units * (double)stride;
  }
  if (max_slots > BATCH_MAX_SLOTS) {
    s.code = DCFR_ERR_UNSUPPORTED;
    s.msg = "a spot's tree needs more than " + std::to_string(BATCH_MAX_SLOTS) + " reach slots";
    return s;
  }
  // Device arrays.
  if (!(s = balloc(regrets, total_store, "batch storage")).ok()) return s;
  if (!(s = balloc(sums, total_store, "batch storage")).ok()) return s;
  BK(cudaMemsetAsync(regrets, 0, std::max<uint64_t>(total_store, 1) * 4, stream));
  BK(cudaMemsetAsync(sums, 0, std::max<uint64_t>(total_store, 1) * 4, stream));
  if (!(s = balloc(vals, vals_off, "batch value rows")).ok()) return s;
  if (!(s = balloc(reach, reach_off, "batch reach rows")).ok()) return s;
  BK(cudaMemsetAsync(vals, 0, std::max<uint64_t>(vals_off, 1) * 4, stream));
  BK(cudaMemsetAsync(reach, 0, std::max<uint64_t>(reach_off, 1) * 4, stream));
  if (!(s = upload(hc1, h1, "batch hands")).ok()) return s;
  if (!(s = upload(hc2, h2, "batch hands")).ok()) return s;
  if (!(s = upload(same, hs, "batch hands")).ok()) return s;
  if (!(s = upload(roots, hroot, "batch root rows")).ok()) return s;
  if (!(s = balloc(root_out, hroot.size(), "batch root rows")).ok()) return s;
  if (!(s = upload(boards, hb, "batch boards")).ok()) return s;
  if (!(s = upload(down, hdown, "batch plan")).ok()) return s;
  if (!(s = upload(up, hup, "batch plan")).ok()) return s;
  if (!(s = upload(term, hterm, "batch plan")).ok()) return s;
  if (!(s = upload(d_spots, spots, "batch plan")).ok()) return s;
  std::vector<uint32_t> nat(count), lpt(count);
  std::iota(nat.begin(), nat.end(), 0u);
  lpt = nat;
  std::stable_sort(lpt.begin(), lpt.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  if (!(s = upload(order_nat, nat, "batch order")).ok()) return s;
  if (!(s = upload(order_lpt, lpt, "batch order")).ok()) return s;
  // Strength tables and scan layouts, per spot (its board and fold layouts).
  if (!(s = balloc(tables, (size_t)count * 2 * tstride, "batch strength tables")).ok()) return s;
  if (!(s = balloc(tcount, (size_t)count * 2, "batch strength tables")).ok()) return s;
  const size_t nl = (size_t)count * 2 * 2;
  if (!(s = balloc(cat, nl * cstride, "batch scan layouts")).ok()) return s;
  if (!(s = balloc(seg, nl * FAST_SEGS, "batch scan layouts")).ok()) return s;
  if (!(s = balloc(rec, nl * tstride, "batch scan layouts")).ok()) return s;
  for (int i = 0; i < count; i++) {
    const SpotD& S = spots[i];
    const uint8_t* a0 = hc1 + S.hands;
    const uint8_t* b0 = hc2 + S.hands;
    const uint8_t* a1 = hc1 + S.hands + S.stride;
    const uint8_t* b1 = hc2 + S.hands + S.stride;
    EntryD* tb = tables + (size_t)i * 2 * tstride;
    uint32_t* tc = tcount + (size_t)i * 2;
    launch_strength(boards + (size_t)i * 5, 1, a0, b0, a1, b1, S.n[0], S.n[1], tb, tc, tstride, stream);
    launch_fast_layouts(tb, tc, tstride, 1, a0, b0, a1, b1, S.n[0], S.n[1], cat + (size_t)S.layout * 2 * cstride,
                        seg + (size_t)S.layout * 2 * FAST_SEGS, rec + (size_t)S.layout * 2 * tstride, cstride,
                        stream);
  }
  BK(cudaGetLastError());
  if (!(s = balloc(counter, 1, "batch counter")).ok()) return s;
  if (!(s = balloc(work, 1, "batch counter")).ok()) return s;
  BK(cudaMemsetAsync(counter, 0, 4, stream));
  BK(cudaMemsetAsync(work, 0, 4, stream));
  if (!(s = ensure_discounts(1024)).ok()) return s;
  // Shared memory: allow every kernel the device's opt-in maximum.
  int optin = 0;
  BK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  for (int mode : {M_CFR, M_BR, M_AVG})
    for (int m : {4, 8, MAX_ACTIONS})
      BK(cudaFuncSetAttribute(batch_kernel_ptr(mode, m), cudaFuncAttributeMaxDynamicSharedMemorySize, optin));
  // Default tuning until autotune: the most resident warps that fit.
  tuning.warps = 0;
  for (int w = 1; w <= BATCH_MAX_THREADS / 32; w++) {
    const size_t smem = BatchSmem(max_slots, max_stride, cstride, tstride, w).total;
    if (smem > (size_t)optin) break;
    int b = 0;
    BK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel_ptr(M_CFR, maxa), w * 32, smem));
    if (b > 0 && w * b >= tuning.warps * tuning.blocks_per_sm) {
      tuning.warps = w;
      tuning.blocks_per_sm = b;
    }
  }
  if (tuning.warps == 0) {
    s.code = DCFR_ERR_UNSUPPORTED;
    s.msg = "batched kernel: a spot's layout does not fit in shared memory";
    return s;
  }
  tuning.iterations_per_launch = 25;
  tuning.longest_first = 1;
  BK(cudaStreamSynchronize(stream));
  return Status();
}

BatchArgs Batch::Impl::args(int mode, uint32_t iters, bool lpt) const {
  BatchArgs B;
  B.regrets = regrets;
  B.sums = sums;
  B.reach = reach;
  B.vals = vals;
  B.root_out = root_out;
  B.hc1 = hc1;
  B.hc2 = hc2;
  B.same = same;
  B.roots = roots;
  B.cat = cat;
  B.seg = seg;
  B.rec = rec;
  B.down = down;
  B.up = up;
  B.term = term;
  B.spots = d_spots;
  B.order = lpt ? order_lpt : order_nat;
  B.nspots = (int)spots.size();
  B.disc_table = disc;
  B.disc_len = disc_len;
  B.counter = counter;
  B.work = work;
  B.cstride = cstride;
  B.tstride = tstride;
  B.max_slots = max_slots;
  B.max_stride = max_stride;
  B.iters = (int)iters;
  (void)mode;
  return B;
}

// One persistent launch: `iters` CFR iterations of every spot (mode M_CFR),
// or one best-response / average traversal pair (M_BR, M_AVG); then the
// iteration counter advances and the work counter resets.
Status Batch::Impl::launch(int mode, uint32_t iters, const dcfr_batch_tuning& t) {
  const BatchArgs B = args(mode, iters, t.longest_first != 0);
  const size_t smem = BatchSmem(max_slots, max_stride, cstride, tstride, t.warps).total;
  const int blocks = std::min<int>((int)spots.size(), sms * std::max(t.blocks_per_sm, 1));
  void* params[] = {(void*)&B};
  BK(cudaLaunchKernel(batch_kernel_ptr(mode, maxa), dim3((unsigned)blocks), dim3((unsigned)(t.warps * 32)), params,
                      smem, stream));
  batch_advance_kernel<<<1, 1, 0, stream>>>(counter, mode == M_CFR ? iters : 0u, work);
  BK(cudaGetLastError());
  launches += 2;
  return Status();
}

Status Batch::Impl::capture(uint32_t iters) {
  if (graph && graph_iters == iters) return Status();
  if (graph) {
    cudaGraphExecDestroy(graph);
    graph = nullptr;
  }
  cudaGraph_t g;
  BK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
  Status s = launch(M_CFR, iters, tuning);
  cudaError_t e = cudaStreamEndCapture(stream, &g);
  launches -= 2;
  if (!s.ok()) return s;
  BK(e);
  BK(cudaGraphInstantiate(&graph, g, 0));
  cudaGraphDestroy(g);
  graph_iters = iters;
  return Status();
}

Status Batch::Impl::run(uint32_t n) {
  Status s;
  if (!(s = ensure_discounts(iterations + n + 1)).ok()) return s;
  const uint32_t k = std::max<uint32_t>(tuning.iterations_per_launch, 1);
  if (!(s = capture(k)).ok()) return s;
  BK(cudaEventRecord(ev0, stream));
  uint32_t done = 0;
  while (n - done >= k) {
    BK(cudaGraphLaunch(graph, stream));
    launches += 2;
    done += k;
  }
  if (done < n) {
    if (!(s = launch(M_CFR, n - done, tuning)).ok()) return s;
  }
  BK(cudaEventRecord(ev1, stream));
  BK(cudaEventSynchronize(ev1));
  float ms = 0.0f;
  BK(cudaEventElapsedTime(&ms, ev0, ev1));
  last_ms = ms;
  iterations += n;
  return Status();
}

Batch::Batch() : impl_(new Impl()) {}
Batch::~Batch() = default;

Status Batch::create(const dcfr_config* cfgs, int count, std::unique_ptr<Batch>& out) {
  Status s;
  if (count <= 0) {
    s.code = DCFR_ERR_INVALID_ARG;
    s.msg = "a batch has at least one spot";
    return s;
  }
  std::unique_ptr<Batch> b(new Batch());
  if (!(s = b->impl_->init(cfgs, count)).ok()) return s;
  out = std::move(b);
  return Status();
}

int Batch::count() const { return (int)impl_->spots.size(); }
uint32_t Batch::iterations() const { return impl_->iterations; }
double Batch::last_iterate_ms() const { return impl_->last_ms; }
uint64_t Batch::kernel_launches() const { return impl_->launches; }
dcfr_batch_tuning Batch::tuning() const { return impl_->tuning; }

double Batch::iteration_bytes() const {
  double b = 0.0;
  for (const Game& g : impl_->games)
    b += 20.0 * (double)g.storage_len + 2.0 * (double)g.nodes.size() * 4.0 * ((double)g.n[0] + (double)g.n[1]);
  return b;
}

Status Batch::iterate(uint32_t n) { return impl_->run(n); }

Status Batch::set_tuning(const dcfr_batch_tuning& t) {
  Status s;
  const size_t smem = BatchSmem(impl_->max_slots, impl_->max_stride, impl_->cstride, impl_->tstride, t.warps).total;
  int dev = 0, optin = 0;
  BK(cudaGetDevice(&dev));
  BK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (t.warps < 1 || t.warps > BATCH_MAX_THREADS / 32 || smem > (size_t)optin || t.iterations_per_launch < 1) {
    s.code = DCFR_ERR_INVALID_ARG;
    s.msg = "batch tuning: warps, shared memory or iterations per launch out of range";
    return s;
  }
  int b = 0;
  BK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel_ptr(M_CFR, impl_->maxa), t.warps * 32, smem));
  dcfr_batch_tuning u = t;
  u.blocks_per_sm = std::max(1, std::min(t.blocks_per_sm > 0 ? t.blocks_per_sm : b, b));
  impl_->tuning = u;
  if (impl_->graph) {
    cudaGraphExecDestroy(impl_->graph);
    impl_->graph = nullptr;
  }
  return Status();
}

// The project's autotuner: times each candidate (warps per block, blocks
// per SM, iterations per launch, longest-first or natural order) on
// `trial_iterations` iterations from a snapshot of the storage, restores the
// snapshot and the iteration counter after every trial, and keeps the
// fastest candidate.
Status Batch::autotune(uint32_t trial_iterations, dcfr_batch_tuning& best) {
  Impl& I = *impl_;
  Status s;
  const uint64_t n = std::max<uint64_t>(I.total_store, 1);
  float *r0 = nullptr, *s0 = nullptr;
  if (!(s = balloc(r0, n, "autotune snapshot")).ok()) return s;
  if (!(s = balloc(s0, n, "autotune snapshot")).ok()) {
    bfree(r0);
    return s;
  }
  BK(cudaMemcpyAsync(r0, I.regrets, n * 4, cudaMemcpyDeviceToDevice, I.stream));
  BK(cudaMemcpyAsync(s0, I.sums, n * 4, cudaMemcpyDeviceToDevice, I.stream));
  const uint32_t t_saved = I.iterations;
  const dcfr_batch_tuning saved = I.tuning;
  int dev = 0, optin = 0;
  BK(cudaGetDevice(&dev));
  BK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  std::vector<dcfr_batch_tuning> cands;
  const uint32_t trial = std::max<uint32_t>(trial_iterations, 1);
  for (int w = 1; w <= BATCH_MAX_THREADS / 32; w++) {
    const size_t smem = BatchSmem(I.max_slots, I.max_stride, I.cstride, I.tstride, w).total;
    if (smem > (size_t)optin) break;
    int b = 0;
    BK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel_ptr(M_CFR, I.maxa), w * 32, smem));
    if (b <= 0 || w < 2) continue;
    for (uint32_t ipl : {trial, std::max<uint32_t>(trial / 5, 1u)})
      for (int lpt : {1, 0}) {
        dcfr_batch_tuning t{};
        t.warps = w;
        t.blocks_per_sm = b;
        t.iterations_per_launch = ipl;
        t.longest_first = lpt;
        cands.push_back(t);
      }
  }
  double best_ms = 1e300;
  best = saved;
  for (const dcfr_batch_tuning& t : cands) {
    if (!(s = set_tuning(t)).ok()) break;
    if (!(s = I.run(trial)).ok()) break;
    const double ms = I.last_ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = I.tuning;
    }
    BK(cudaMemcpyAsync(I.regrets, r0, n * 4, cudaMemcpyDeviceToDevice, I.stream));
    BK(cudaMemcpyAsync(I.sums, s0, n * 4, cudaMemcpyDeviceToDevice, I.stream));
    BK(cudaMemcpyAsync(I.counter, &t_saved, 4, cudaMemcpyHostToDevice, I.stream));
    BK(cudaStreamSynchronize(I.stream));
    I.iterations = t_saved;
  }
  bfree(r0);
  bfree(s0);
  if (!s.ok()) {
    set_tuning(saved);
    return s;
  }
  best.trial_ms = best_ms;
  best.candidates = (int)cands.size();
  return set_tuning(best);
}

Status Batch::root_values(int mode, std::vector<double>& out) {
  Impl& I = *impl_;
  Status s;
  if (!(s = I.launch(mode, 1, I.tuning)).ok()) return s;
  std::vector<float> rows(I.spots.empty() ? 0 : (size_t)I.spots.back().root + 2 * I.spots.back().stride);
  BK(cudaMemcpyAsync(rows.data(), I.root_out, rows.size() * 4, cudaMemcpyDeviceToHost, I.stream));
  BK(cudaStreamSynchronize(I.stream));
  out.assign(I.spots.size() * 2, 0.0);
  for (size_t i = 0; i < I.spots.size(); i++) {
    const SpotD& S = I.spots[i];
    const Game& g = I.games[i];
    for (int p = 0; p < 2; p++) {
      double acc = -0.0;
      for (int h = 0; h < g.n[p]; h++)
        acc += (double)rows[S.root + (size_t)p * S.stride + h] * (double)g.weights[p][h];
      out[2 * i + p] = acc;
    }
  }
  return Status();
}

Status Batch::exploitability(double* out) {
  std::vector<double> br, ev;
  Status s = root_values(M_BR, br);
  if (!s.ok()) return s;
  bool raked = false;
  for (const Game& g : impl_->games) raked |= g.cfg.rake_rate > 0.0 && g.cfg.rake_cap > 0.0;
  if (raked && !(s = root_values(M_AVG, ev)).ok()) return s;
  for (size_t i = 0; i < impl_->games.size(); i++) {
    const dcfr_config& c = impl_->games[i].cfg;
    if (c.rake_rate > 0.0 && c.rake_cap > 0.0)
      out[i] = ((br[2 * i] - ev[2 * i]) + (br[2 * i + 1] - ev[2 * i + 1])) / 2.0;
    else
      out[i] = (br[2 * i] + br[2 * i + 1]) / 2.0;
  }
  return Status();
}

Status Batch::storage_len(int spot, uint64_t& len) const {
  if (spot < 0 || spot >= count()) return Status{DCFR_ERR_INVALID_ARG, "spot index out of range"};
  len = impl_->games[spot].storage_len;
  return Status();
}

Status Batch::download(int spot, float* regrets, float* sums) {
  Impl& I = *impl_;
  if (spot < 0 || spot >= count()) return Status{DCFR_ERR_INVALID_ARG, "spot index out of range"};
  const Game& g = I.games[spot];
  const SpotD& S = I.spots[spot];
  std::vector<float> r(I.spot_len[spot]), sm(I.spot_len[spot]);
  BK(cudaMemcpyAsync(r.data(), I.regrets + S.store, r.size() * 4, cudaMemcpyDeviceToHost, I.stream));
  BK(cudaMemcpyAsync(sm.data(), I.sums + S.store, sm.size() * 4, cudaMemcpyDeviceToHost, I.stream));
  BK(cudaStreamSynchronize(I.stream));
  for (uint32_t v = 0; v < g.nodes.size(); v++) {
    const GNode& nd = g.nodes[v];
    if (nd.kind != N_PLAYER) continue;
    const int q = nd.player, n = g.n[q], hq = S.hp[q];
    for (int a = 0; a < nd.nchild; a++) {
      if (regrets)
        std::memcpy(regrets + nd.ref_offset + (size_t)a * n, r.data() + I.node_off[spot][v] + (size_t)a * hq, n * 4);
      if (sums)
        std::memcpy(sums + nd.ref_offset + (size_t)a * n, sm.data() + I.node_off[spot][v] + (size_t)a * hq, n * 4);
    }
  }
  return Status();
}

}  // namespace dcfr
