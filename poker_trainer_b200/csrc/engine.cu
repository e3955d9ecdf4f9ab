// Device engine of libdcfr (see engine.hpp): planning, device memory, graph
// capture, the solve loop (Solver::run_solve, crates/solver/src/lib.rs:594-642),
// exploitability (cfr.rs:482-502) and queries (lib.rs:735-912).
#include "engine.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <unordered_map>

namespace dcfr {

Status cuda_status(cudaError_t e, const char* what) {
  Status s;
  if (e == cudaSuccess) return s;
  s.code = (e == cudaErrorMemoryAllocation) ? DCFR_ERR_OUT_OF_MEMORY : DCFR_ERR_CUDA;
  s.msg = std::string(what) + ": " + cudaGetErrorString(e);
  return s;
}

#define CK(call)                                  \
  do {                                            \
    Status _s = cuda_status((call), #call);       \
    if (!_s.ok()) return _s;                      \
  } while (0)

template <class T>
static Status dalloc(T*& p, size_t count, const char* what) {
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
static void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

static inline int pad8(int n) { return (n + 7) & ~7; }

Plan::~Plan() {
  dfree(d_down);
  dfree(d_up);
  dfree(d_groups);
  dfree(d_lanes);
  dfree(d_tasks);
  dfree(d_fast);
  dfree(d_units);
  dfree(d_panels);
  dfree(d_leaves);
  dfree(d_trees);
  dfree(d_fdown);
  dfree(d_fup);
}

// DcfrParams -> Discount (cfr.rs:86-106), host f64 pow as the reference.
static DiscountD discount_for(uint32_t t, const dcfr_params& prm) {
  uint32_t tm = t < 1 ? 1 : t;
  double prev = (double)(tm - 1);
  double pa = std::pow(prev, prm.alpha);
  float neg = 0.0f;
  if (!prm.beta_clip) {
    double pb = std::pow(prev, prm.beta);
    neg = (float)(pb / (pb + 1.0));
  }
  double since = (double)tm - 1.0;
  if (prm.restart_average) {
    uint32_t t0 = tm - 1;
    uint32_t p4 = t0 == 0 ? 0 : (1u << ((31u - (uint32_t)__builtin_clz(t0)) & ~1u));
    since = (double)(t0 - p4);
  }
  DiscountD d;
  d.pos = (float)(pa / (pa + 1.0));
  d.neg = neg;
  d.strat = (float)std::pow(since / (since + 1.0), prm.gamma);
  d.reach_weighted = prm.unweighted_average ? 0 : 1;
  return d;
}

DiscountD discount_of(uint32_t t, const dcfr_params& prm) { return discount_for(t, prm); }

// next_check_gap (lib.rs:158-172).
static uint32_t next_gap(bool has_prev, uint32_t t0, double e0, uint32_t t, double e, double target,
                         uint32_t max_gap) {
  uint32_t min_gap = std::max(max_gap / 4, 1u);
  if (!has_prev) return max_gap;
  if (!(e < e0 && e > target && t > t0 && target > 0.0)) return max_gap;
  double k = std::log(e0 / e) / std::log((double)t / (double)t0);
  double predicted = (double)t * std::pow(e / target, 1.0 / k);
  double gap = std::ceil(predicted - (double)t);
  if (!std::isfinite(gap)) return max_gap;
  double gg = gap > 0.0 ? gap : 0.0;
  uint32_t gu = gg >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)gg;
  return std::min(std::max(gu, min_gap), max_gap);
}

// Milliseconds since t0 (host clock), for the setup profile.
static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

Status Engine::create(const dcfr_config& cfg, std::unique_ptr<Engine>& out) {
  const auto t0 = std::chrono::steady_clock::now();
  std::unique_ptr<Engine> e(new Engine());
  Status s;
  if (cfg.precision != DCFR_PRECISION_FAST && cfg.precision != DCFR_PRECISION_EXACT) {
    s.code = DCFR_ERR_INVALID_ARG;
    s.msg = "precision must be DCFR_PRECISION_FAST or DCFR_PRECISION_EXACT";
    return s;
  }
  e->fast_ = cfg.precision == DCFR_PRECISION_FAST;
  s.code = build_game(cfg, e->g, s.msg, true);
  if (!s.ok()) return s;
  e->setup.game_ms = ms_since(t0);
  s = e->init();
  if (!s.ok()) return s;
  e->setup.create_ms = ms_since(t0);
  out = std::move(e);
  return Status();
}

Status Engine::create_depth_limited(const dcfr_config& cfg, dcfr_mlp* net, int leaf_street,
                                    std::unique_ptr<Engine>& out) {
  std::unique_ptr<Engine> e(new Engine());
  Status s;
  if (!net) return Status{DCFR_ERR_INVALID_ARG, "depth-limited solve: NULL network"};
  if (cfg.board_len != 3 || cfg.root.street != DCFR_FLOP || leaf_street != DCFR_TURN)
    return Status{DCFR_ERR_UNSUPPORTED, "depth-limited solves take a flop root cut at the turn deal"};
  if (cfg.precision != DCFR_PRECISION_FAST)
    return Status{DCFR_ERR_UNSUPPORTED, "depth-limited solves run in fast precision"};
  if (cfg.rake_rate > 0.0 && cfg.rake_cap > 0.0)
    return Status{DCFR_ERR_UNSUPPORTED, "depth-limited solves take unraked games"};
  e->fast_ = true;
  s.code = build_game(cfg, e->g, s.msg, true, leaf_street);
  if (!s.ok()) return s;
  if (e->g.compressed) return Status{DCFR_ERR_UNSUPPORTED, "depth-limited solves run f32 storage"};
  e->net_ = net;
  if (!(s = e->init()).ok()) return s;
  if (!(s = e->init_leaves()).ok()) return s;
  out = std::move(e);
  return Status();
}

Engine::~Engine() {
  if (stream_) cudaStreamSynchronize(stream_);
  free_graphs();
  full_[0].reset();
  full_[1].reset();
  dfree(regrets_);
  dfree(sums_);
  dfree(rq_);
  dfree(sq_);
  dfree(rscale_);
  dfree(sscale_);
  dfree(reach_);
  dfree(vals_);
  dfree(alive_);
  dfree(root_rows_);
  dfree(root_out_);
  for (int q = 0; q < 2; q++) {
    dfree(hc1_[q]);
    dfree(hc2_[q]);
    dfree(same_[q]);
  }
  dfree(perm_);
  dfree(chance_cards_);
  dfree(iso_);
  dfree(tables_);
  dfree(table_count_);
  dfree(progs_);
  dfree(prog_count_);
  dfree(posmap_);
  for (int q = 0; q < 2; q++) {
    dfree(fold_prog_[q]);
    dfree(emit_rec_[q]);
  }
  dfree(warp_scratch_);
  dfree(group_scratch_);
  dfree(counters_);
  dfree(term_counter_);
  dfree(fcat_);
  dfree(fseg_);
  dfree(frec_);
  for (int q = 0; q < 2; q++) {
    dfree(leaf_reach_[q]);
    dfree(combos_[q]);
  }
  dfree(leaf_x_);
  dfree(leaf_cards_);
  dfree(sblk_);
  dfree(reach64_);
  dfree(vals64_);
  dfree(root_rows64_);
  dfree(disc_table_);
  dfree(cur_disc_);
  dfree(counter_);
  for (cudaEvent_t e : prof_events_) cudaEventDestroy(e);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (stream_) cudaStreamDestroy(stream_);
}

void Engine::free_graphs() {
  if (iter_graph_) cudaGraphExecDestroy(iter_graph_);
  if (br_graph_) cudaGraphExecDestroy(br_graph_);
  if (avg_graph_) cudaGraphExecDestroy(avg_graph_);
  iter_graph_ = br_graph_ = avg_graph_ = nullptr;
  if (prof_exec_) cudaGraphExecDestroy(prof_exec_);
  if (prof_graph_) cudaGraphDestroy(prof_graph_);
  prof_exec_ = nullptr;
  prof_graph_ = nullptr;
  marks_.clear();
}

int Engine::isomorphic_pairs() const {
  int k = 0;
  for (int i = 0; i < 6; i++) k += g.sym[i];
  return k;
}

// Algorithmic bytes of one DCFR iteration: every decision node is once the
// traverser's (regret read + write) and once the opponent's (regret read,
// strategy-sum read + write): 20 B per storage cell in f32, 10 B with 16-bit
// storage; plus, per traversal, one opponent-reach row read and one value
// row write per node.
double Engine::iteration_bytes() const {
  double cells = (double)g.storage_len * (compressed_ ? 0.5 : 1.0);
  double nodes = (double)g.nodes.size();
  return 20.0 * cells + 2.0 * nodes * 4.0 * ((double)g.n[0] + (double)g.n[1]);
}

Status Engine::init() {
  auto t0 = std::chrono::steady_clock::now();
  auto phase = [&](double& slot) {
    slot += ms_since(t0);
    t0 = std::chrono::steady_clock::now();
  };
  last_exploitability = INFINITY;
  CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  CK(cudaEventCreate(&ev0_));
  CK(cudaEventCreate(&ev1_));
  CK(terminal_kernel_setup());
  hp_[0] = pad8(g.n[0]);
  hp_[1] = pad8(g.n[1]);
  stride_ = std::max(hp_[0], hp_[1]);
  const size_t N = g.nodes.size();

  // Storage layout: one [actions][hp_q] block per decision node, in the
  // reference's node order (Node::offset, tree.rs:462, 468).
  const std::vector<uint32_t> players = players_in_storage_order(g);
  gpu_off_.assign(N, 0);
  gpu_len_ = 0;
  for (uint32_t v : players) {
    gpu_off_[v] = gpu_len_;
    gpu_len_ += (uint64_t)g.nodes[v].nchild * (uint64_t)hp_[g.nodes[v].player];
  }
  Status s;
  compressed_ = g.compressed;

  tstride_ = std::max(g.n[0], g.n[1]);
  pstride_ = (2 * tstride_ + TERM_CHUNK - 1) / TERM_CHUNK * TERM_CHUNK;
  // Hands.
  for (int q = 0; q < 2; q++) {
    std::vector<uint8_t> a(hp_[q], 255), b(hp_[q], 255);
    std::vector<uint32_t> sm(hp_[q], NO);
    for (int i = 0; i < g.n[q]; i++) {
      a[i] = g.c1[q][i];
      b[i] = g.c2[q][i];
      sm[i] = g.same[q][i];
    }
    if (!(s = dalloc(hc1_[q], hp_[q], "hands")).ok()) return s;
    if (!(s = dalloc(hc2_[q], hp_[q], "hands")).ok()) return s;
    if (!(s = dalloc(same_[q], hp_[q], "hands")).ok()) return s;
    CK(cudaMemcpy(hc1_[q], a.data(), hp_[q], cudaMemcpyHostToDevice));
    CK(cudaMemcpy(hc2_[q], b.data(), hp_[q], cudaMemcpyHostToDevice));
    CK(cudaMemcpy(same_[q], sm.data(), hp_[q] * 4, cudaMemcpyHostToDevice));
    if (fast_) continue;
    // The player's hands in hand order as sweep steps (fold sums) and per-hand
    // emit records (terminal.cu).
    const int npad = (g.n[q] + TERM_CHUNK - 1) / TERM_CHUNK * TERM_CHUNK;
    if (!(s = dalloc(fold_prog_[q], npad, "hands")).ok()) return s;
    if (!(s = dalloc(emit_rec_[q], g.n[q], "hands")).ok()) return s;
    launch_hand_program(hc1_[q], hc2_[q], same_[q], g.n[q], npad, fold_prog_[q], emit_rec_[q], stream_);
    CK(cudaGetLastError());
  }
  {
    std::vector<uint16_t> perm((size_t)12 * stride_, 0);
    for (int q = 0; q < 2; q++)
      for (int pr = 0; pr < 6; pr++)
        for (size_t h = 0; h < g.perm[q][pr].size(); h++) perm[(size_t)(q * 6 + pr) * stride_ + h] = g.perm[q][pr][h];
    if (!(s = dalloc(perm_, perm.size(), "perm")).ok()) return s;
    CK(cudaMemcpy(perm_, perm.data(), perm.size() * 2, cudaMemcpyHostToDevice));
  }
  // Chance cards and isomorphic references.
  {
    std::vector<uint8_t> cc;
    std::vector<IsoRefD> iso;
    cc_off_.assign(g.chance.size(), 0);
    iso_first_.assign(g.chance.size(), 0);
    for (uint32_t v = 0; v < N; v++) {
      const GNode& nd = g.nodes[v];
      if (nd.kind != N_CHANCE) continue;
      cc_off_[nd.index] = (uint32_t)cc.size();
      for (uint32_t c = nd.first; c < nd.first + nd.nchild; c++) cc.push_back((uint8_t)g.nodes[c].card);
      iso_first_[nd.index] = (uint32_t)iso.size();
      const ChanceIso& ci = g.chance[nd.index];
      for (size_t r = 0; r < ci.ci.size(); r++) iso.push_back(IsoRefD{ci.ci[r], ci.pair[r], 0});
    }
    if (!(s = dalloc(chance_cards_, cc.size(), "chance cards")).ok()) return s;
    if (!cc.empty()) CK(cudaMemcpy(chance_cards_, cc.data(), cc.size(), cudaMemcpyHostToDevice));
    if (!(s = dalloc(iso_, iso.size(), "iso refs")).ok()) return s;
    if (!iso.empty()) CK(cudaMemcpy(iso_, iso.data(), iso.size() * sizeof(IsoRefD), cudaMemcpyHostToDevice));
  }
  phase(setup.device_ms);
  // Strength tables, built on the device.
  {
    const int nb = (int)g.boards.size();
    if (!(s = dalloc(tables_, (size_t)std::max(nb, 1) * 2 * tstride_, "strength tables")).ok()) return s;
    if (!(s = dalloc(table_count_, (size_t)std::max(nb, 1) * 2, "strength tables")).ok()) return s;
    if (nb > 0) {
      std::vector<uint8_t> bc((size_t)nb * 5);
      for (int b = 0; b < nb; b++)
        for (int k = 0; k < 5; k++) bc[(size_t)b * 5 + k] = (uint8_t)g.boards[b][k];
      uint8_t* d_boards = nullptr;
      if (!(s = dalloc(d_boards, bc.size(), "boards")).ok()) return s;
      CK(cudaMemcpy(d_boards, bc.data(), bc.size(), cudaMemcpyHostToDevice));
      launch_strength(d_boards, nb, hc1_[0], hc2_[0], hc1_[1], hc2_[1], g.n[0], g.n[1], tables_, table_count_,
                      tstride_, stream_);
      CK(cudaGetLastError());
      if (!fast_) {
        // Sweep programs (terminal.cu): per board, traverser and pass.
        if (!(s = dalloc(progs_, (size_t)nb * 6 * pstride_, "sweep programs")).ok()) return s;
        if (!(s = dalloc(prog_count_, (size_t)nb * 6, "sweep programs")).ok()) return s;
        if (!(s = dalloc(posmap_, (size_t)nb * 6 * tstride_, "sweep programs")).ok()) return s;
        launch_programs(tables_, table_count_, tstride_, progs_, prog_count_, posmap_, pstride_, nb, stream_);
        CK(cudaGetLastError());
      }
      CK(cudaStreamSynchronize(stream_));
      cudaFree(d_boards);
    }
    if (fast_ && !(s = ensure_fast_layouts()).ok()) return s;
  }
  phase(setup.tables_ms);
  // Plans for the two traversals of an iteration, built on two host threads
  // (build_plan only reads the game and host-side fields of the engine)
  // while this thread allocates and clears the storage on the device.
  {
    Status ps[2];
    for (int p = 0; p < 2; p++) full_[p].reset(new Plan());
    std::thread t1([&]() { ps[1] = build_plan(0, 1, *full_[1]); });
    std::thread t0([&]() { ps[0] = build_plan(0, 0, *full_[0]); });
    const Status sa = alloc_storage();
    t0.join();
    t1.join();
    if (!sa.ok()) return sa;
    for (int p = 0; p < 2; p++) {
      if (!ps[p].ok()) return ps[p];
      max_slots_ = std::max<uint64_t>(max_slots_, full_[p]->nslots);
    }
  }
  phase(setup.plans_ms);
  // Rows.
  if (!(s = dalloc(reach_, (size_t)max_slots_ * stride_, "reach rows")).ok()) return s;
  if (!(s = dalloc(vals_, (size_t)N * stride_, "value rows")).ok()) return s;
  if (!(s = dalloc(alive_, (size_t)max_slots_, "liveness flags")).ok()) return s;
  CK(cudaMemsetAsync(reach_, 0, (size_t)max_slots_ * stride_ * 4, stream_));
  CK(cudaMemsetAsync(vals_, 0, (size_t)N * stride_ * 4, stream_));
  {
    std::vector<float> rr((size_t)2 * stride_, 0.0f);
    for (int p = 0; p < 2; p++)
      for (int i = 0; i < g.n[p ^ 1]; i++) rr[(size_t)p * stride_ + i] = g.weights[p ^ 1][i];
    if (!(s = dalloc(root_rows_, rr.size(), "root rows")).ok()) return s;
    CK(cudaMemcpy(root_rows_, rr.data(), rr.size() * 4, cudaMemcpyHostToDevice));
    if (!(s = dalloc(root_out_, rr.size(), "root rows")).ok()) return s;
  }
  phase(setup.rows_ms);
  // Terminal scratch, sized for the largest terminal launch of the two plans.
  if (!fast_) {
    for (int p = 0; p < 2; p++)
      for (const Plan::Wave& w : full_[p]->waves) {
        wave_tasks_ = std::max<int>(wave_tasks_, (int)w.count);
        wave_groups_ = std::max<int>(wave_groups_, (int)w.groups);
      }
    warp_scratch_floats_ = (size_t)(pstride_ + 1) * 32 + (size_t)stride_ * 32;
    if (!(s = dalloc(warp_scratch_, (size_t)std::max(wave_tasks_, 1) * warp_scratch_floats_, "terminal scratch")).ok())
      return s;
    if (!(s = dalloc(group_scratch_, (size_t)std::max(wave_groups_, 1) * 2 * tstride_ * 32, "terminal scratch")).ok())
      return s;
    if (!(s = dalloc(counters_, (size_t)std::max(wave_groups_, 1), "terminal scratch")).ok()) return s;
    CK(cudaMemsetAsync(counters_, 0, (size_t)std::max(wave_groups_, 1) * 4, stream_));
  }
  for (int p = 0; p < 2; p++)
    if (!(s = upload_plan(*full_[p])).ok()) return s;
  phase(setup.plans_ms);
  // Default f32 terminal kernel: two warps per terminal where both
  // traversals have at least four terminal tasks per SM (measured faster there
  // than both the warp and the block kernel); the warp or block kernel for
  // fewer tasks (a river subgame's few dozen terminals: each gets a whole
  // block). The rule depends on the plans and the SM count only.
  if (term_group_auto_) {
    const size_t enough = (size_t)4 * (size_t)term_sms_;
    term_group_ = full_[0]->h_fast.size() >= enough && full_[1]->h_fast.size() >= enough;
  }
  if (!(s = dalloc(cur_disc_, 1, "discounts")).ok()) return s;
  if (!(s = dalloc(counter_, 1, "counter")).ok()) return s;
  CK(cudaMemsetAsync(counter_, 0, 4, stream_));
  if (!(s = ensure_discounts(1024)).ok()) return s;
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// Storage in the layout of Engine::init, zeroed: f32 regrets and strategy
// sums, or 16-bit values with a scale of each kind per decision node.
Status Engine::alloc_storage() {
  Status s;
  if (compressed_) {
    // Storage::Compressed (storage.rs:92-97): 16-bit values, a scale of
    // each kind per decision node (its ordinal, the reference's slot).
    const size_t slots = std::max<size_t>(g.player_nodes, 1);
    if (!(s = dalloc(rq_, gpu_len_, "storage")).ok()) return s;
    if (!(s = dalloc(sq_, gpu_len_, "storage")).ok()) return s;
    if (!(s = dalloc(rscale_, slots, "storage scales")).ok()) return s;
    if (!(s = dalloc(sscale_, slots, "storage scales")).ok()) return s;
    CK(cudaMemsetAsync(rq_, 0, gpu_len_ * 2, stream_));
    CK(cudaMemsetAsync(sq_, 0, gpu_len_ * 2, stream_));
    CK(cudaMemsetAsync(rscale_, 0, slots * 4, stream_));
    CK(cudaMemsetAsync(sscale_, 0, slots * 4, stream_));
  } else {
    if (!(s = dalloc(regrets_, gpu_len_, "storage")).ok()) return s;
    if (!(s = dalloc(sums_, gpu_len_, "storage")).ok()) return s;
    CK(cudaMemsetAsync(regrets_, 0, gpu_len_ * 4, stream_));
    CK(cudaMemsetAsync(sums_, 0, gpu_len_ * 4, stream_));
  }
  return Status();
}

// Scan layouts of the fast terminal kernel (terminal_fast.cu): the boards'
// strength tables, then the fold layout. Built in init for fast precision,
// and on first use by the FP64 best-response oracle in exact precision.
Status Engine::ensure_fast_layouts() {
  if (fcat_) return Status();
  Status s;
  const int nb = (int)g.boards.size();
  fcstride_ = (3 * tstride_ + 7) / 8 * 8;
  femax_ = fast_emax(tstride_);
  const size_t nl = (size_t)(nb + 1) * 2;
  if (!(s = dalloc(fcat_, nl * fcstride_, "scan layouts")).ok()) return s;
  if (!(s = dalloc(fseg_, nl * FAST_SEGS, "scan layouts")).ok()) return s;
  if (!(s = dalloc(frec_, nl * tstride_, "scan layouts")).ok()) return s;
  launch_fast_layouts(tables_, table_count_, tstride_, nb, hc1_[0], hc2_[0], hc1_[1], hc2_[1], g.n[0], g.n[1], fcat_,
                      fseg_, frec_, fcstride_, stream_);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(stream_));
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int per_sm = fast_blocks_per_sm(stride_, femax_, fcstride_, tstride_);
  if (per_sm <= 0) {
    s.code = DCFR_ERR_CUDA;
    s.msg = "terminal kernel: shared-memory layout does not fit an SM";
    return s;
  }
  fast_blocks_ = sms * per_sm;
  // The f32 solve's terminal kernel: a warp per terminal for short hand
  // lists, a block-wide scan per terminal for long ones (measured fastest);
  // DCFR_TERMINAL_KERNEL selects another one (panel, panel4, panel8, warp,
  // block) for comparisons.
  const char* sel = std::getenv("DCFR_TERMINAL_KERNEL");
  const std::string want = sel ? sel : (tstride_ <= WARP_TERMINAL_MAX_HANDS ? "warp" : "block");
  term_kernel_ = want == "warp" || want == "warpdyn" || want == "group" ? TK_WARP
                 : want == "block" || want == "blockdyn" ? TK_BLOCK
                                                         : TK_PANEL;
  term_dynamic_ = want == "warpdyn" || want == "blockdyn";
  if (term_dynamic_ && term_kernel_ == TK_WARP) {
    int bps = 0;
    dyn_warps_ = warp_terminal_dyn_setup(stride_, fcstride_, tstride_, 16, bps);
    dyn_blocks_ = sms * bps;
    if (dyn_warps_ <= 0) term_dynamic_ = false;
  }
  if (term_dynamic_ && !(s = dalloc(term_counter_, 1, "terminal counter")).ok()) return s;
  // Two warps per terminal (terminal_group.cu): explicitly, or by default
  // where both traversals have enough terminal tasks (decided in init once
  // the plans are built).
  term_sms_ = sms;
  {
    int bps = 0;
    group_groups_ = group_terminal_setup(stride_, fcstride_, tstride_, bps);
    group_blocks_ = sms * bps;
  }
  term_group_ = want == "group" && group_groups_ > 0;
  term_group_auto_ = sel == nullptr && group_groups_ > 0;
  if (term_kernel_ == TK_PANEL) {
    const int o0 = 1, o1 = 0;  // opponent of traverser 0 and 1
    panel_T_ = panel_E_ = panel_blocks_ = 0;
    for (int T : {8, 4}) {
      if ((want == "panel4" && T != 4) || (want == "panel8" && T != 8)) continue;
      // One setup per traverser: the shared-memory footprint depends on both
      // players' padded hand counts; the larger one sets the limit.
      int b0 = 0, b1 = 0;
      const int e0 = panel_terminal_setup(hp_[o0], hp_[0], fcstride_, tstride_, T, b0);
      const int e1 = panel_terminal_setup(hp_[o1], hp_[1], fcstride_, tstride_, T, b1);
      if (e0 > 0 && e1 > 0 && e0 == e1) {
        panel_T_ = T;
        panel_E_ = e0;
        panel_blocks_ = sms * std::min(b0, b1);
        break;
      }
    }
    if (panel_T_ == 0) term_kernel_ = tstride_ <= WARP_TERMINAL_MAX_HANDS ? TK_WARP : TK_BLOCK;
  }
  for (int k = 0; k < 2; k++) {
    int bps = 0;
    term_warps_[k] = warp_terminal_setup(stride_, fcstride_, tstride_, k ? 8 : 4, 16, bps);
    term_blocks_[k] = sms * bps;
    if (term_warps_[k] <= 0) {
      s.code = DCFR_ERR_CUDA;
      s.msg = "warp terminal kernel: shared-memory layout does not fit an SM";
      return s;
    }
  }
  return Status();
}

// Level-synchronous plan of one traversal (see plan.hpp).
Status Engine::build_plan(uint32_t root, int p, Plan& plan) {
  plan.p = p;
  plan.root = root;
  const int o = p ^ 1;
  std::vector<std::vector<DownTask>> down;
  std::vector<std::vector<UpTask>> up;
  std::vector<int> dmax, umax;
  struct SdLane {
    uint32_t kind, board;
    TermLane lane;
  };
  std::vector<SdLane> sd;
  std::vector<TermLane> folds[2];
  uint32_t next_slot = 1;
  // Breadth-first queue (popped at qh). An entry carries what the node
  // inherits from its parent: its reach slot, chance layer, and the parent's
  // fused segment, depth in it and depth in a wide segment (NONE32: none).
  struct QItem {
    uint32_t v, depth, slot, layer, ptree, ptdepth, psdepth;
  };
  std::vector<QItem> q;
  size_t qh = 0;
  const size_t NN = g.nodes.size();
  // Every street's decision subtree is a segment: the traversal's root and
  // each child of a chance node. A segment runs fused (one block,
  // fused_*_kernel) or level by level. Chance nodes sit between segments;
  // layer(v) counts the chance nodes above v, so a traversal runs segment
  // layer 0, chance layer 0, segment layer 1, ... down, and the reverse up.
  auto segment_root = [&](uint32_t v) {
    const GNode& nd = g.nodes[v];
    return nd.kind == N_PLAYER && (v == root || (nd.parent != NO && g.nodes[nd.parent].kind == N_CHANCE));
  };
  // A segment runs fused only where its layer has at least
  // FUSE_MIN_SEGMENTS segments (one block each fills the GPU) and it has at
  // most FUSE_MAX_NODES decision nodes. Others (the traversal's root
  // segment, wide segments) run level by level: one launch per depth, with
  // many blocks per node.
  constexpr uint32_t FUSE_MAX_NODES = 48, FUSE_MIN_SEGMENTS = 16;
  // The traversal's nodes in id order. build_game appends a node's children
  // after it, so ids grow from parent to child and a pass in id order visits
  // every parent before its children (the reverse pass, children first).
  std::vector<uint32_t> sub;
  if (root == 0) {
    sub.resize(NN);
    for (uint32_t v = 0; v < NN; v++) sub[v] = v;
  } else {
    std::vector<uint32_t> st{root};
    while (!st.empty()) {
      const uint32_t v = st.back();
      st.pop_back();
      sub.push_back(v);
      const GNode& nd = g.nodes[v];
      if (nd.kind == N_PLAYER || nd.kind == N_CHANCE)
        for (uint32_t i = 0; i < nd.nchild; i++) st.push_back(nd.first + i);
    }
    std::sort(sub.begin(), sub.end());
  }
  // Decision nodes per segment (keyed by the segment's root) and segments
  // per chance layer.
  std::vector<uint32_t> seg_size(NN, 0);
  std::vector<uint32_t> layer_segments;
  size_t nplayer = 0, nshow = 0, nfold = 0;  // the traversal's nodes by kind (capacities)
  {
    std::vector<uint32_t> seg_of(NN, 0), lay(NN, 0);
    for (const uint32_t v : sub) {
      const GNode& nd = g.nodes[v];
      uint32_t seg = root, layer = 0;
      if (v != root) {
        const uint32_t u = nd.parent;
        if (g.nodes[u].kind == N_PLAYER) {
          seg = seg_of[u];
          layer = lay[u];
        } else {
          seg = v;
          layer = lay[u] + 1;
        }
      }
      lay[v] = layer;
      nshow += nd.kind == N_SHOWDOWN;
      nfold += nd.kind == N_FOLD;
      if (nd.kind != N_PLAYER) continue;
      nplayer++;
      uint32_t rr = seg;
      if (segment_root(v)) {
        rr = v;
        if (layer_segments.size() <= layer) layer_segments.resize(layer + 1, 0);
        layer_segments[layer]++;
      }
      seg_size[rr]++;
      seg_of[v] = rr;
    }
  }
  auto fused_segment = [&](uint32_t v, uint32_t layer) {
    return seg_size[v] <= FUSE_MAX_NODES && layer < layer_segments.size() &&
           layer_segments[layer] >= FUSE_MIN_SEGMENTS;
  };
  std::vector<std::vector<std::vector<DownTask>>> sdown;  // wide segments: [layer][depth]
  std::vector<std::vector<std::vector<UpTask>>> sup;
  // Fused segments' tasks in discovery (breadth-first) order with their
  // segment and depth in it; bucketed by segment below.
  struct FDown {
    uint32_t tree, depth;
    DownTask t;
  };
  struct FUp {
    uint32_t tree, depth;
    UpTask t;
  };
  std::vector<FDown> fdown;
  std::vector<FUp> fup;
  std::vector<uint32_t> tree_layer;
  int fmaxa = 0;
  q.reserve(sub.size());
  fdown.reserve(nplayer);
  fup.reserve(nplayer);
  sd.reserve(nshow);
  folds[1].reserve(nfold);
  q.push_back({root, 0, 0, 0, NONE32, 0, NONE32});
  const double hp = g.half_pot, norm = g.norm;
  uint64_t count = 0;
  while (qh < q.size()) {
    // The queue holds the next nodes already: request their records ahead
    // of use (breadth-first order jumps across the node array).
    if (qh + 24 < q.size()) {
      const uint32_t w = q[qh + 24].v;
      __builtin_prefetch(&g.nodes[w]);
      __builtin_prefetch(&gpu_off_[w]);
      __builtin_prefetch(&seg_size[w]);
    }
    if (qh + 8 < q.size()) {
      const GNode& wn = g.nodes[q[qh + 8].v];
      if (wn.kind == N_PLAYER || wn.kind == N_CHANCE) __builtin_prefetch(&g.nodes[wn.first]);
    }
    const QItem it = q[qh++];
    const uint32_t v = it.v, depth = it.depth;
    count++;
    const GNode& nd = g.nodes[v];
    const uint32_t sv = it.slot;
    const uint32_t layer = it.layer;
    const uint32_t clayer = layer + (nd.kind == N_CHANCE ? 1u : 0u);  // the children's
    uint32_t tree = NONE32, tdepth = 0, sdepth = NONE32;
    if (segment_root(v) && fused_segment(v, layer)) {
      tree = (uint32_t)tree_layer.size();
      tree_layer.push_back(layer);
    } else if (segment_root(v)) {
      sdepth = 0;
    } else if (nd.kind == N_PLAYER && it.ptree != NONE32) {
      tree = it.ptree;
      tdepth = it.ptdepth + 1;
    }
    if (tree != NONE32 && nd.kind == N_PLAYER) {
      // Inside a fused river subtree (no chance nodes below the river).
      bool own = nd.player == p;
      uint32_t first_slot = own ? sv : next_slot;
      if (!own) next_slot += nd.nchild;
      for (uint32_t i = 0; i < nd.nchild; i++)
        q.push_back({nd.first + i, depth + 1, own ? sv : first_slot + i, clayer, tree, tdepth, NONE32});
      if (nd.nchild > MAX_ACTIONS) {
        Status s;
        s.code = DCFR_ERR_INVALID_ARG;
        s.msg = "a decision node has more than 16 actions";
        return s;
      }
      // `cards` of a decision node's tasks: its scale slot (compressed storage).
      if (!own)
        fdown.push_back({tree, tdepth, DownTask{D_OPP_SPLIT, sv, first_slot, nd.nchild, gpu_off_[v], nd.index, 0.0f}});
      fup.push_back({tree, tdepth, UpTask{own ? (uint32_t)U_OWN : (uint32_t)U_OPP_SUM, sv, v, nd.first, nd.nchild,
                                          first_slot, gpu_off_[v], nd.index, 0, 0, 0}});
      fmaxa = std::max<int>(fmaxa, (int)nd.nchild);
    } else if (nd.kind == N_PLAYER || nd.kind == N_CHANCE) {
      // Chance nodes, by layer (decision nodes all belong to segments).
      const uint32_t depth = layer;
      if (down.size() <= depth) {
        down.resize(depth + 1);
        up.resize(depth + 1);
        dmax.resize(depth + 1, 0);
        umax.resize(depth + 1, 0);
      }
      if (nd.nchild > MAX_ACTIONS && nd.kind == N_PLAYER) {
        Status s;
        s.code = DCFR_ERR_INVALID_ARG;
        s.msg = "a decision node has more than 16 actions";
        return s;
      }
      bool own = nd.kind == N_PLAYER && nd.player == p;
      uint32_t first_slot = own ? sv : next_slot;
      if (!own) next_slot += nd.nchild;
      if (nd.kind == N_PLAYER && sdepth == NONE32) sdepth = it.psdepth + 1;
      for (uint32_t i = 0; i < nd.nchild; i++)
        q.push_back({nd.first + i, depth + 1, own ? sv : first_slot + i, clayer, tree, tdepth, sdepth});
      if (nd.kind == N_PLAYER) {
        // A node of a wide segment: level by level.
        const uint32_t sd = sdepth;
        if (sdown.size() <= layer) {
          sdown.resize(layer + 1);
          sup.resize(layer + 1);
        }
        if (sdown[layer].size() <= sd) {
          sdown[layer].resize(sd + 1);
          sup[layer].resize(sd + 1);
        }
        if (!own)
          sdown[layer][sd].push_back(DownTask{D_OPP_SPLIT, sv, first_slot, nd.nchild, gpu_off_[v], nd.index, 0.0f});
        sup[layer][sd].push_back(UpTask{own ? (uint32_t)U_OWN : (uint32_t)U_OPP_SUM, sv, v, nd.first, nd.nchild,
                                        first_slot, gpu_off_[v], nd.index, 0, 0, 0});
      } else {
        DownTask t{D_CHANCE_SPLIT, sv, first_slot, nd.nchild, 0, cc_off_[nd.index], nd.factor};
        down[depth].push_back(t);
        UpTask u{U_CHANCE_SUM, sv, v, nd.first, nd.nchild, first_slot, 0, cc_off_[nd.index], iso_first_[nd.index],
                 (uint32_t)g.chance[nd.index].ci.size(), 0};
        up[depth].push_back(u);
      }
    } else if (nd.kind == N_LEAF) {
      // Depth-limited cut: valued by the leaf-value network (leaf.cu).
      const Game::Leaf& lf = g.leaves[nd.index];
      plan.h_leaves.push_back(LeafTask{nd.index, sv, v, 0, (float)lf.pot, (float)lf.stack});
    } else {
      // Terminal. Batched evaluation (river.rs) iff the terminal sits below a
      // river decision node inside this traversal (cfr.rs:282-284).
      bool batch = v != root && nd.parent != NO && g.nodes[nd.parent].kind == N_PLAYER &&
                   g.nodes[nd.parent].street == DCFR_RIVER;
      TermLane L{sv, v, NONE32, 0, 0.0, 0.0, 0.0, 0.0};
      if (nd.kind == N_FOLD) {
        // fold_payoff (cfr.rs:226-235).
        int f = nd.player;
        double val = f == p ? -(hp + (double)nd.invest[p]) : hp + (double)nd.invest[f] - (double)nd.rake;
        L.a = val * norm;
        if (batch) {
          // A fold next to a showdown under the traverser's own decision
          // shares its reach and is read off the showdown sweep
          // (river.rs:190-240).
          const GNode& par = g.nodes[nd.parent];
          bool paired = false;
          if (par.player == p)
            for (uint32_t c = par.first; c < par.first + par.nchild; c++)
              if (g.nodes[c].kind == N_SHOWDOWN) paired = true;
          if (paired) continue;
        }
        folds[batch ? 1 : 0].push_back(L);
      } else {
        // showdown_payoffs (cfr.rs:239-246).
        double rake = (double)nd.rake;
        L.a = (hp + (double)nd.invest[o] - rake) * norm;
        L.b = -(hp + (double)nd.invest[p]) * norm;
        L.c = 0.5 * ((double)(nd.invest[o] - nd.invest[p]) - rake) * norm;
        if (batch) {
          const GNode& par = g.nodes[nd.parent];
          if (par.player == p)
            for (uint32_t c = par.first; c < par.first + par.nchild; c++)
              if (g.nodes[c].kind == N_FOLD) {
                const GNode& fn = g.nodes[c];
                int f = fn.player;
                double val = f == p ? -(hp + (double)fn.invest[p]) : hp + (double)fn.invest[f] - (double)fn.rake;
                L.frow = c;
                L.d = val * norm;
              }
        }
        sd.push_back(SdLane{batch ? (uint32_t)T_SHOWDOWN_BATCH : (uint32_t)T_SHOWDOWN_SCALAR, nd.index, L});
      }
    }
  }
  plan.nodes = count;
  plan.nslots = next_slot;
  // Fused subtrees: down tasks in BFS order with a barrier at each new level,
  // up tasks deepest level first.
  plan.h_trees.clear();
  plan.h_fdown.clear();
  plan.h_fup.clear();
  plan.fused_maxa = fmaxa;
  // Segments by layer: one fused launch per layer.
  const uint32_t ntrees = (uint32_t)tree_layer.size();
  std::vector<uint32_t> order(ntrees);
  for (size_t t = 0; t < order.size(); t++) order[t] = (uint32_t)t;
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return tree_layer[a] < tree_layer[b]; });
  // Each segment's tasks, discovery order kept (counting sort by segment).
  std::vector<uint32_t> fd_off(ntrees + 1, 0), fu_off(ntrees + 1, 0);
  for (const FDown& x : fdown) fd_off[x.tree + 1]++;
  for (const FUp& x : fup) fu_off[x.tree + 1]++;
  for (uint32_t t = 0; t < ntrees; t++) {
    fd_off[t + 1] += fd_off[t];
    fu_off[t + 1] += fu_off[t];
  }
  std::vector<uint32_t> fd_idx(fdown.size()), fu_idx(fup.size());
  {
    std::vector<uint32_t> fill(fd_off.begin(), fd_off.end() - 1);
    for (size_t i = 0; i < fdown.size(); i++) fd_idx[fill[fdown[i].tree]++] = (uint32_t)i;
    std::vector<uint32_t> ufill(fu_off.begin(), fu_off.end() - 1);
    for (size_t i = 0; i < fup.size(); i++) fu_idx[ufill[fup[i].tree]++] = (uint32_t)i;
  }
  plan.h_fdown.reserve(fdown.size());
  plan.h_fup.reserve(fup.size());
  plan.h_trees.reserve(ntrees);
  plan.tree_layers.clear();
  for (uint32_t t : order) {
    const uint32_t l = tree_layer[t];
    if (plan.tree_layers.size() <= l) plan.tree_layers.resize(l + 1, {(uint32_t)plan.h_trees.size(), 0u});
    plan.tree_layers[l].second++;
    FusedTree F{(uint32_t)plan.h_fdown.size(), 0, (uint32_t)plan.h_fup.size(), 0};
    uint32_t prev = 0;
    for (uint32_t i = fd_off[t]; i < fd_off[t + 1]; i++) {
      const FDown& x = fdown[fd_idx[i]];
      DownTask T = x.t;
      if (i > fd_off[t] && x.depth != prev) T.kind |= LEVEL_BREAK;
      prev = x.depth;
      plan.h_fdown.push_back(T);
    }
    // Up tasks deepest level first, discovery order within a level: the
    // segment's levels (depth non-decreasing in discovery order) reversed.
    uint32_t e = fu_off[t + 1];
    while (e > fu_off[t]) {
      uint32_t b = e - 1;
      const uint32_t d = fup[fu_idx[b]].depth;
      while (b > fu_off[t] && fup[fu_idx[b - 1]].depth == d) b--;
      for (uint32_t i = b; i < e; i++) plan.h_fup.push_back(fup[fu_idx[i]].t);
      e = b;
    }
    F.down_count = (uint32_t)(plan.h_fdown.size() - F.down_first);
    F.up_count = (uint32_t)(plan.h_fup.size() - F.up_first);
    plan.h_trees.push_back(F);
  }
  // Flatten levels.
  plan.h_down.clear();
  plan.h_up.clear();
  plan.down.assign(down.size(), Plan::Level());
  plan.up.assign(up.size(), Plan::Level());
  // Within a level, tasks by kind (one launch per kind present).
  for (size_t d = 0; d < down.size(); d++) {
    std::stable_sort(down[d].begin(), down[d].end(),
                     [](const DownTask& a, const DownTask& b) { return a.kind < b.kind; });
    std::stable_sort(up[d].begin(), up[d].end(), [](const UpTask& a, const UpTask& b) { return a.kind < b.kind; });
    plan.down[d] = Plan::Level{(uint32_t)plan.h_down.size(), (uint32_t)down[d].size(), dmax[d], {0, 0, 0}};
    for (const DownTask& t : down[d]) plan.down[d].kind_count[t.kind]++;
    plan.h_down.insert(plan.h_down.end(), down[d].begin(), down[d].end());
    plan.up[d] = Plan::Level{(uint32_t)plan.h_up.size(), (uint32_t)up[d].size(), umax[d], {0, 0, 0}};
    for (const UpTask& t : up[d]) plan.up[d].kind_count[t.kind]++;
    plan.h_up.insert(plan.h_up.end(), up[d].begin(), up[d].end());
  }
  // Wide segments: per layer, one level per depth.
  plan.seg_down.assign(sdown.size(), {});
  plan.seg_up.assign(sup.size(), {});
  for (size_t l = 0; l < sdown.size(); l++)
    for (size_t d = 0; d < sdown[l].size(); d++) {
      int maxa = 0;
      for (const DownTask& t : sdown[l][d]) maxa = std::max<int>(maxa, (int)t.nchild);
      plan.seg_down[l].push_back(Plan::Level{(uint32_t)plan.h_down.size(), (uint32_t)sdown[l][d].size(), maxa,
                                             {0, 0, 0}});
      plan.h_down.insert(plan.h_down.end(), sdown[l][d].begin(), sdown[l][d].end());
      maxa = 0;
      for (const UpTask& t : sup[l][d]) maxa = std::max<int>(maxa, (int)t.nchild);
      plan.seg_up[l].push_back(Plan::Level{(uint32_t)plan.h_up.size(), (uint32_t)sup[l][d].size(), maxa, {0, 0, 0}});
      plan.h_up.insert(plan.h_up.end(), sup[l][d].begin(), sup[l][d].end());
    }
  // Exact precision's terminal groups: showdowns by (kind, board), folds by
  // kind, 32 lanes each (fast precision uses h_fast only).
  if (!fast_)
    std::stable_sort(sd.begin(), sd.end(), [](const SdLane& a, const SdLane& b) {
      return a.kind != b.kind ? a.kind < b.kind : a.board < b.board;
    });
  plan.h_groups.clear();
  plan.h_lanes.clear();
  for (size_t i = 0; !fast_ && i < sd.size();) {
    size_t j = i;
    while (j < sd.size() && j - i < 32 && sd[j].kind == sd[i].kind && sd[j].board == sd[i].board) j++;
    TermGroup G{sd[i].kind, sd[i].board, (uint32_t)plan.h_lanes.size(), (uint32_t)(j - i)};
    for (size_t k = i; k < j; k++) plan.h_lanes.push_back(sd[k].lane);
    plan.h_groups.push_back(G);
    i = j;
  }
  for (int b = 0; b < 2 && !fast_; b++)
    for (size_t i = 0; i < folds[b].size(); i += 32) {
      size_t j = std::min(folds[b].size(), i + 32);
      TermGroup G{b ? (uint32_t)T_FOLD_BATCH : (uint32_t)T_FOLD_SCALAR, 0, (uint32_t)plan.h_lanes.size(),
                  (uint32_t)(j - i)};
      for (size_t k = i; k < j; k++) plan.h_lanes.push_back(folds[b][k]);
      plan.h_groups.push_back(G);
    }
  // Fast precision: one task per terminal, grouped by layout. A fold below
  // a river decision node is evaluated on its river board's layout: the
  // opponent hands that layout leaves out hold a board card and have zero
  // reach there, so every integer sum is the same as on the all-hands fold
  // layout, and the board's folds interleave with its showdowns (blocks of
  // the terminal kernels take contiguous task ranges; folds are cheaper).
  // Other folds use the fold layout (index nboards).
  const uint32_t nb = (uint32_t)g.boards.size();
  // Decision node -> the river board below it: passed up from each showdown
  // through its decision-node ancestors (one street segment; every showdown
  // below a decision node of that segment has the same board), children
  // first, then above the traversal's root.
  std::vector<uint32_t> seg_board(NN, NONE32);
  for (size_t i = sub.size(); i-- > 0;) {
    const uint32_t v = sub[i];
    const GNode& nd = g.nodes[v];
    const uint32_t b = nd.kind == N_SHOWDOWN ? nd.index : nd.kind == N_PLAYER ? seg_board[v] : NONE32;
    if (b == NONE32 || nd.parent == NO) continue;
    if (v == root) {
      for (uint32_t u = nd.parent; u != NO && g.nodes[u].kind == N_PLAYER && seg_board[u] == NONE32;
           u = g.nodes[u].parent)
        seg_board[u] = b;
    } else if (g.nodes[nd.parent].kind == N_PLAYER && seg_board[nd.parent] == NONE32) {
      seg_board[nd.parent] = b;
    }
  }
  // Each fold's layout, then per layout the showdowns' and folds' indices
  // (counting sort: the tasks themselves are written once, in final order).
  std::vector<uint32_t> fold_layout(folds[0].size() + folds[1].size(), nb);
  for (size_t i = 0; i < folds[1].size(); i++)
    for (uint32_t u = g.nodes[folds[1][i].row].parent; u != NO && g.nodes[u].kind == N_PLAYER;
         u = g.nodes[u].parent)
      if (seg_board[u] != NONE32) {
        fold_layout[folds[0].size() + i] = seg_board[u];
        break;
      }
  std::vector<uint32_t> s_off(nb + 2, 0), f_off(nb + 2, 0);
  for (const SdLane& x : sd) s_off[x.board + 1]++;
  for (uint32_t l : fold_layout) f_off[l + 1]++;
  for (uint32_t l = 0; l <= nb; l++) {
    s_off[l + 1] += s_off[l];
    f_off[l + 1] += f_off[l];
  }
  std::vector<uint32_t> s_idx(sd.size()), f_idx(fold_layout.size());
  {
    std::vector<uint32_t> fill(s_off.begin(), s_off.end() - 1);
    for (size_t i = 0; i < sd.size(); i++) s_idx[fill[sd[i].board]++] = (uint32_t)i;
    std::vector<uint32_t> ffill(f_off.begin(), f_off.end() - 1);
    for (size_t i = 0; i < fold_layout.size(); i++) f_idx[ffill[fold_layout[i]]++] = (uint32_t)i;
  }
  auto sd_task = [&](uint32_t i) {
    const SdLane& x = sd[i];
    const TermLane& L = x.lane;
    return FastTask{x.kind, x.board, L.slot, L.row, L.frow, {0, 0, 0}, L.a, L.b, L.c, L.d};
  };
  auto fold_task = [&](uint32_t i) {
    const bool b = i >= folds[0].size();
    const TermLane& L = b ? folds[1][i - folds[0].size()] : folds[0][i];
    return FastTask{b ? (uint32_t)T_FOLD_BATCH : (uint32_t)T_FOLD_SCALAR, fold_layout[i], L.slot, L.row, NONE32,
                    {0, 0, 0}, L.a, 0.0, 0.0, 0.0};
  };
  // Within a layout, showdowns and folds are interleaved evenly in chunks of
  // PT tasks (after k chunks, about k |S| / (|S| + |F|) showdown chunks).
  // With the panel kernel a chunk is a panel, all showdowns or all folds.
  plan.h_fast.clear();
  plan.h_fast.reserve(sd.size() + fold_layout.size());
  plan.h_panels.clear();
  const bool panels = fast_ && term_kernel_ == TK_PANEL;
  const size_t PT = panels ? (size_t)panel_T_ : 1;
  for (uint32_t l = 0; l <= nb; l++) {
    const size_t S0 = s_off[l], SN = s_off[l + 1] - S0, F0 = f_off[l], FN = f_off[l + 1] - F0;
    const size_t ns = (SN + PT - 1) / PT, nf = (FN + PT - 1) / PT;
    size_t i = 0, j = 0;
    while (i < ns || j < nf) {
      const bool take_s = j >= nf || (i < ns && i * nf <= j * ns);
      const size_t c = take_s ? i++ : j++;
      const size_t a = c * PT, e = std::min(take_s ? SN : FN, a + PT);
      if (panels) plan.h_panels.push_back(PanelD{(uint32_t)plan.h_fast.size(), (uint32_t)(e - a), l, 0});
      for (size_t k = a; k < e; k++)
        plan.h_fast.push_back(take_s ? sd_task(s_idx[S0 + k]) : fold_task(f_idx[F0 + k]));
    }
  }
  // Units of the warp terminal kernel: maximal runs of tasks on one layout
  // (h_fast is ordered by layout).
  plan.h_units.clear();
  for (size_t i = 0; i < plan.h_fast.size();) {
    size_t j = i;
    while (j < plan.h_fast.size() && plan.h_fast[j].board == plan.h_fast[i].board) j++;
    plan.h_units.push_back(TermUnit{plan.h_fast[i].board, (uint32_t)i, (uint32_t)(j - i), 0});
    i = j;
  }
  // Terminal tasks: one warp per fold group; per showdown group, the
  // ascending and descending passes and, when a terminal has a paired fold,
  // the paired fold's pass. Launches ("waves") are bounded in tasks and in
  // showdown groups (scratch).
  plan.h_tasks.clear();
  plan.waves.clear();
  Plan::Wave wave;
  auto close_wave = [&]() {
    if (wave.count) plan.waves.push_back(wave);
    wave = Plan::Wave();
    wave.first = (uint32_t)plan.h_tasks.size();
  };
  wave.first = 0;
  for (size_t gi = 0; gi < plan.h_groups.size(); gi++) {
    const TermGroup& G = plan.h_groups[gi];
    if (G.kind == T_FOLD_SCALAR || G.kind == T_FOLD_BATCH) {
      if (wave.count + 1 > (uint32_t)MAX_WAVE_TASKS) close_wave();
      plan.h_tasks.push_back(TermTask{R_FOLD, (uint32_t)gi, 0, 0});
      wave.count += 1;
      continue;
    }
    bool paired = false;
    for (uint32_t k = 0; k < G.count; k++) paired |= plan.h_lanes[G.first + k].frow != NONE32;
    const uint32_t need = paired ? 3 : 2;
    if (wave.count + need > (uint32_t)MAX_WAVE_TASKS || wave.groups + 1 > (uint32_t)MAX_WAVE_GROUPS) close_wave();
    const uint32_t wg = wave.groups++;
    plan.h_tasks.push_back(TermTask{R_ASC, (uint32_t)gi, wg, 0});
    plan.h_tasks.push_back(TermTask{R_DESC, (uint32_t)gi, wg, 0});
    if (paired) plan.h_tasks.push_back(TermTask{R_PAIRED, (uint32_t)gi, wg, 0});
    wave.count += need;
  }
  close_wave();
  int kernels = 0;
  int tree_launches = 0;
  for (auto& tl : plan.tree_layers) tree_launches += tl.second > 0;
  for (auto& l : plan.down) kernels += l.count > 0;
  for (auto& l : plan.up) kernels += l.count > 0;
  kernels += 2 * tree_launches;
  int seg_down_launches = 0, seg_up_launches = 0;
  for (auto& ls : plan.seg_down)
    for (auto& l : ls) seg_down_launches += l.count > 0;
  for (auto& ls : plan.seg_up)
    for (auto& l : ls) seg_up_launches += l.count > 0;
  kernels += seg_down_launches + seg_up_launches;
  const int term_kernels = fast_ ? (plan.h_fast.empty() ? 0 : 1) : (int)plan.waves.size();
  kernels += term_kernels;
  kernels += 1;  // the traversal's start (liveness flags, root row)
  plan.kernels = kernels;
  // Per class: launches and compulsory bytes of one CFR traversal (rows of
  // n floats, f32 storage).
  for (int c = 0; c < DCFR_KERNEL_CLASSES; c++) {
    plan.class_kernels[c] = 0;
    plan.class_bytes[c] = 0.0;
  }
  for (auto& l : plan.down) plan.class_kernels[DCFR_KERNEL_DOWN] += l.count > 0;
  for (auto& l : plan.up) plan.class_kernels[DCFR_KERNEL_UP] += l.count > 0;
  plan.class_kernels[DCFR_KERNEL_DOWN] += tree_launches + seg_down_launches;
  plan.class_kernels[DCFR_KERNEL_UP] += tree_launches + seg_up_launches;
  plan.class_kernels[DCFR_KERNEL_TERMINAL] = term_kernels;
  plan.class_kernels[DCFR_KERNEL_OTHER] = 1;
  const double np_ = g.n[p], no_ = g.n[o];
  for (const std::vector<DownTask>* v : {&plan.h_down, &plan.h_fdown})
    for (const DownTask& t : *v)
      // Opponent split: reach row in, k rows out, regrets read, sums read and
      // written (2-byte values with compressed storage).
      plan.class_bytes[DCFR_KERNEL_DOWN] += (t.kind & KIND_MASK) == D_OPP_SPLIT
                                                ? 4.0 * no_ * (1.0 + t.nchild) + (compressed_ ? 6.0 : 12.0) * no_ * t.nchild
                                                : 4.0 * no_ * (1.0 + t.nchild);
  for (const std::vector<UpTask>* v : {&plan.h_up, &plan.h_fup})
    for (const UpTask& t : *v)
      plan.class_bytes[DCFR_KERNEL_UP] += t.kind == U_OWN
                                              ? 4.0 * np_ * (t.nchild + 1.0) + (compressed_ ? 4.0 : 8.0) * np_ * t.nchild
                                              : 4.0 * np_ * (t.nchild + 1.0);
  // Per terminal: one reach row read, one value row written, and the paired
  // fold's row.
  for (const FastTask& t : plan.h_fast)
    plan.class_bytes[DCFR_KERNEL_TERMINAL] += 4.0 * (no_ + np_) + (t.frow != NONE32 ? 4.0 * np_ : 0.0);
  return Status();
}

Status Engine::upload_plan(Plan& plan) {
  Status s;
  if (!(s = dalloc(plan.d_down, plan.h_down.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_up, plan.h_up.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_groups, plan.h_groups.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_lanes, plan.h_lanes.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_tasks, plan.h_tasks.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_fast, plan.h_fast.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_units, plan.h_units.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_leaves, plan.h_leaves.size(), "plan")).ok()) return s;
  if (!plan.h_leaves.empty())
    CK(cudaMemcpy(plan.d_leaves, plan.h_leaves.data(), plan.h_leaves.size() * sizeof(LeafTask),
                  cudaMemcpyHostToDevice));
  if (!plan.h_units.empty())
    CK(cudaMemcpy(plan.d_units, plan.h_units.data(), plan.h_units.size() * sizeof(TermUnit), cudaMemcpyHostToDevice));
  if (!(s = dalloc(plan.d_panels, plan.h_panels.size(), "plan")).ok()) return s;
  if (!plan.h_panels.empty())
    CK(cudaMemcpy(plan.d_panels, plan.h_panels.data(), plan.h_panels.size() * sizeof(PanelD),
                  cudaMemcpyHostToDevice));
  if (!(s = dalloc(plan.d_trees, plan.h_trees.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_fdown, plan.h_fdown.size(), "plan")).ok()) return s;
  if (!(s = dalloc(plan.d_fup, plan.h_fup.size(), "plan")).ok()) return s;
  if (!plan.h_trees.empty()) {
    CK(cudaMemcpy(plan.d_trees, plan.h_trees.data(), plan.h_trees.size() * sizeof(FusedTree), cudaMemcpyHostToDevice));
    if (!plan.h_fdown.empty())
      CK(cudaMemcpy(plan.d_fdown, plan.h_fdown.data(), plan.h_fdown.size() * sizeof(DownTask),
                    cudaMemcpyHostToDevice));
    if (!plan.h_fup.empty())
      CK(cudaMemcpy(plan.d_fup, plan.h_fup.data(), plan.h_fup.size() * sizeof(UpTask), cudaMemcpyHostToDevice));
  }
  if (!plan.h_fast.empty())
    CK(cudaMemcpy(plan.d_fast, plan.h_fast.data(), plan.h_fast.size() * sizeof(FastTask), cudaMemcpyHostToDevice));
  if (!plan.h_tasks.empty())
    CK(cudaMemcpy(plan.d_tasks, plan.h_tasks.data(), plan.h_tasks.size() * sizeof(TermTask), cudaMemcpyHostToDevice));
  if (!plan.h_down.empty())
    CK(cudaMemcpy(plan.d_down, plan.h_down.data(), plan.h_down.size() * sizeof(DownTask), cudaMemcpyHostToDevice));
  if (!plan.h_up.empty())
    CK(cudaMemcpy(plan.d_up, plan.h_up.data(), plan.h_up.size() * sizeof(UpTask), cudaMemcpyHostToDevice));
  if (!plan.h_groups.empty())
    CK(cudaMemcpy(plan.d_groups, plan.h_groups.data(), plan.h_groups.size() * sizeof(TermGroup),
                  cudaMemcpyHostToDevice));
  if (!plan.h_lanes.empty())
    CK(cudaMemcpy(plan.d_lanes, plan.h_lanes.data(), plan.h_lanes.size() * sizeof(TermLane), cudaMemcpyHostToDevice));
  return Status();
}

void Engine::row_args(int p, RowArgs& A) const {
  A.regrets = regrets_;
  A.sums = sums_;
  A.rq = rq_;
  A.sq = sq_;
  A.rscale = rscale_;
  A.sscale = sscale_;
  A.compressed = compressed_ ? 1 : 0;
  A.reach = reach_;
  A.vals = vals_;
  A.alive = alive_;
  for (int q = 0; q < 2; q++) {
    A.hc1[q] = hc1_[q];
    A.hc2[q] = hc2_[q];
    A.n[q] = g.n[q];
    A.hp[q] = hp_[q];
  }
  A.perm = perm_;
  A.chance_cards = chance_cards_;
  A.iso = iso_;
  A.disc = cur_disc_;
  A.stride = stride_;
  A.p = p;
}

void Engine::term_args(int p, TermArgs& A) const {
  A.reach = reach_;
  A.vals = vals_;
  A.alive = alive_;
  A.warp_scratch = warp_scratch_;
  A.warp_scratch_floats = warp_scratch_floats_;
  A.group_scratch = group_scratch_;
  A.counters = counters_;
  A.tables = tables_;
  A.table_count = table_count_;
  A.progs = progs_;
  A.prog_count = prog_count_;
  A.posmap = posmap_;
  for (int q = 0; q < 2; q++) {
    A.fold_prog[q] = fold_prog_[q];
    A.emit_rec[q] = emit_rec_[q];
  }
  A.pstride = pstride_;
  for (int q = 0; q < 2; q++) {
    A.hc1[q] = hc1_[q];
    A.hc2[q] = hc2_[q];
    A.same[q] = same_[q];
    A.n[q] = g.n[q];
    A.hp[q] = hp_[q];
  }
  A.stride = stride_;
  A.tstride = tstride_;
  A.nmax = tstride_;
  A.p = p;
}

void Engine::fast_args(int p, FastArgs& A) const {
  A.reach = reach_;
  A.vals = vals_;
  A.alive = alive_;
  A.cat = fcat_;
  A.seg = fseg_;
  A.rec = frec_;
  A.same = same_[p];
  A.cstride = fcstride_;
  A.tstride = tstride_;
  A.emax = femax_;
  for (int q = 0; q < 2; q++) {
    A.n[q] = g.n[q];
    A.hp[q] = hp_[q];
  }
  A.stride = stride_;
  A.p = p;
}

// Enqueues one traversal: liveness reset, root row, down levels, terminals,
// up levels (deepest first); the root's value row is copied to root_out.
void Engine::enqueue_traversal(const Plan& plan, int mode, const float* root_row, float* root_out, bool advance) {
  const int p = plan.p, o = p ^ 1;
  launch_traversal_start(alive_, (int)plan.nslots, reach_, root_row, stride_, advance ? counter_ : nullptr,
                         disc_table_, disc_len_, cur_disc_, stream_);
  mark(DCFR_KERNEL_OTHER);
  RowArgs A;
  row_args(p, A);
  const size_t layers = std::max({plan.tree_layers.size(), plan.down.size(), plan.seg_down.size()});
  // Down: segment layer l (fused segments, then wide ones level by level),
  // then the chance nodes of layer l.
  for (size_t l = 0; l < layers; l++) {
    if (l < plan.tree_layers.size() && plan.tree_layers[l].second)
      launch_fused_down(mode, plan.fused_maxa, A, plan.d_trees + plan.tree_layers[l].first,
                        (int)plan.tree_layers[l].second, plan.d_fdown, hp_[o], stream_);
    if (l < plan.seg_down.size())
      for (const Plan::Level& lv : plan.seg_down[l])
        if (lv.count) launch_down(mode, lv.maxa, A, plan.d_down + lv.first, (int)lv.count, hp_[o], stream_);
    if (l < plan.down.size() && plan.down[l].count)
      launch_down(mode, plan.down[l].maxa, A, plan.d_down + plan.down[l].first, (int)plan.down[l].count, hp_[o],
                  stream_);
  }
  mark(DCFR_KERNEL_DOWN);
  if (fast_) {
    if (!plan.h_fast.empty()) {
      FastArgs F;
      fast_args(p, F);
      // Panels of T terminals per block; or (a selectable alternative) a
      // warp per terminal for short rows and one block-wide scan per
      // terminal for long rows.
      // Two warps per terminal (the default where there are enough tasks,
      // for short and long hand lists alike) comes first.
      if (term_group_)
        launch_group_terminal(F, plan.d_fast, plan.d_units, (int)plan.h_units.size(), (int)plan.h_fast.size(),
                              group_groups_, group_blocks_, stream_);
      else if (term_kernel_ == TK_PANEL)
        launch_panel_terminal(F, plan.d_fast, plan.d_panels, (int)plan.h_panels.size(), panel_T_, panel_E_,
                              panel_blocks_, stream_);
      else if (term_kernel_ == TK_WARP && term_dynamic_)
        launch_warp_terminal_dyn(F, plan.d_fast, plan.d_units, (int)plan.h_units.size(), (int)plan.h_fast.size(),
                                 dyn_warps_, dyn_blocks_, term_counter_, stream_);
      else if (term_kernel_ == TK_WARP)
        launch_warp_terminal(F, plan.d_fast, plan.d_units, (int)plan.h_units.size(), (int)plan.h_fast.size(),
                             term_warps_[0], term_blocks_[0],
                             stream_);
      else if (term_dynamic_)
        launch_fast_terminal_dyn(F, plan.d_fast, (int)plan.h_fast.size(), fast_blocks_, term_counter_, stream_);
      else
        launch_fast_terminal(F, plan.d_fast, (int)plan.h_fast.size(), fast_blocks_, stream_);
    }
  } else if (!plan.waves.empty()) {
    TermArgs T;
    term_args(p, T);
    for (const Plan::Wave& w : plan.waves)
      launch_terminal(T, plan.d_groups, plan.d_lanes, plan.d_tasks + w.first, (int)w.count, stream_);
  }
  enqueue_leaves(plan);
  mark(DCFR_KERNEL_TERMINAL);
  // Up: the chance nodes of layer l (their children are done), then segment
  // layer l.
  for (size_t l = layers; l-- > 0;) {
    if (l < plan.up.size() && plan.up[l].count)
      launch_up(mode, plan.up[l].maxa, A, plan.d_up + plan.up[l].first, (int)plan.up[l].count, hp_[p], stream_);
    if (l < plan.seg_up.size())
      for (size_t d = plan.seg_up[l].size(); d-- > 0;) {
        const Plan::Level& lv = plan.seg_up[l][d];
        if (lv.count) launch_up(mode, lv.maxa, A, plan.d_up + lv.first, (int)lv.count, hp_[p], stream_);
      }
    if (l < plan.tree_layers.size() && plan.tree_layers[l].second)
      launch_fused_up(mode, plan.fused_maxa, A, plan.d_trees + plan.tree_layers[l].first,
                      (int)plan.tree_layers[l].second, plan.d_fup, hp_[p], stream_);
  }
  mark(DCFR_KERNEL_UP);
  if (root_out)
    cudaMemcpyAsync(root_out, vals_ + (size_t)plan.root * stride_, (size_t)stride_ * 4, cudaMemcpyDeviceToDevice,
                    stream_);
}

// Depth-limited solves: buffers of the leaf evaluation, and both players'
// ranges at the leaves from one pass of average-strategy traversals (the
// strategy sums are zero at creation: uniform strategies).
Status Engine::init_leaves() {
  Status s;
  const int L = (int)g.leaves.size();
  std::vector<uint8_t> cards;
  uint64_t used = 0;
  for (int c : g.board) used |= 1ull << c;
  for (int c = 0; c < 52; c++)
    if (!(used >> c & 1)) cards.push_back((uint8_t)c);
  leaf_nc_ = (int)cards.size();
  // Chance factor of the deal at the leaves, as a chance node's (tree.rs:520-542):
  // 1 / (cards * compatible / available) in f32.
  const float compatible = (float)(52 - (int)g.board.size() - 4);
  leaf_factor_ = 1.0f / ((float)leaf_nc_ * compatible / (float)leaf_nc_);
  int in_dim = 0, out_dim = 0, max_batch = 0;
  if (mlp_shape(net_, &in_dim, &out_dim, &max_batch))
    return Status{DCFR_ERR_INVALID_ARG, "depth-limited solve: invalid network"};
  if (in_dim != 2 * DCFR_NUM_COMBOS + 54 || out_dim != 2 * DCFR_NUM_COMBOS)
    return Status{DCFR_ERR_INVALID_ARG, "leaf network must map 2706 inputs to 2652 outputs"};
  if (max_batch < std::max(L, 1) * leaf_nc_)
    return Status{DCFR_ERR_INVALID_ARG, "leaf network batch is smaller than leaves x dealt cards (" +
                                            std::to_string(L * leaf_nc_) + ")"};
  for (int q = 0; q < 2; q++) {
    if (!(s = dalloc(leaf_reach_[q], (size_t)std::max(L, 1) * stride_, "leaf ranges")).ok()) return s;
    CK(cudaMemsetAsync(leaf_reach_[q], 0, (size_t)std::max(L, 1) * stride_ * 4, stream_));
    std::vector<uint16_t> cb(hp_[q], 0);
    for (int i = 0; i < g.n[q]; i++) cb[i] = g.combos[q][i];
    if (!(s = dalloc(combos_[q], cb.size(), "leaf combos")).ok()) return s;
    CK(cudaMemcpy(combos_[q], cb.data(), cb.size() * 2, cudaMemcpyHostToDevice));
  }
  if (!(s = dalloc(leaf_x_, (size_t)std::max(L, 1) * leaf_nc_ * (2 * DCFR_NUM_COMBOS + 54), "leaf inputs")).ok())
    return s;
  if (!(s = dalloc(leaf_cards_, cards.size(), "leaf cards")).ok()) return s;
  CK(cudaMemcpy(leaf_cards_, cards.data(), cards.size(), cudaMemcpyHostToDevice));
  for (int p = 0; p < 2; p++)
    enqueue_traversal(*full_[p], M_AVG, root_rows_ + (size_t)p * stride_, nullptr);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(stream_));
  return leaf_status_;
}

void Engine::enqueue_leaves(const Plan& plan) {
  if (!net_ || plan.h_leaves.empty()) return;
  const int p = plan.p, o = p ^ 1;
  LeafArgs A;
  A.reach = reach_;
  A.vals = vals_;
  A.alive = alive_;
  for (int q = 0; q < 2; q++) {
    A.leaf_reach[q] = leaf_reach_[q];
    A.combos[q] = combos_[q];
    A.n[q] = g.n[q];
  }
  A.x = leaf_x_;
  A.y = nullptr;
  A.ldy = 0;
  A.cards = leaf_cards_;
  A.nc = leaf_nc_;
  for (int k = 0; k < 3; k++) A.board[k] = g.board[k];
  A.stride = stride_;
  A.p = p;
  A.factor = leaf_factor_;
  A.norm = g.norm;
  const int nl = (int)plan.h_leaves.size();
  launch_leaf_capture(A, plan.d_leaves, nl, stream_);
  launch_leaf_inputs(A, plan.d_leaves, nl, hc1_[0], hc2_[0], hc1_[1], hc2_[1], stream_);
  const float* y = nullptr;
  int ldy = 0;
  if (mlp_enqueue_forward(net_, leaf_x_, (int)g.leaves.size() * leaf_nc_, stream_, &y, &ldy) != DCFR_OK) {
    leaf_status_ = Status{DCFR_ERR_CUDA, "leaf network forward pass failed"};
    return;
  }
  A.y = y;
  A.ldy = ldy;
  launch_leaf_values(A, plan.d_leaves, nl, hc1_[p], hc2_[p], hc1_[o], hc2_[o], hp_[p], stream_);
}

static Status bad_path(const std::string& m);

Status Engine::node_storage(const std::vector<dcfr_step>& path, uint64_t& offset, int& num_actions, int& num_hands) {
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  uint32_t node = 0;
  Status s = walk(path, node, reach, to_canon);
  if (!s.ok()) return s;
  const GNode& nd = g.nodes[node];
  if (nd.kind != N_PLAYER) return bad_path("not a decision node");
  offset = nd.ref_offset;
  num_actions = nd.nchild;
  num_hands = g.n[nd.player];
  return Status();
}

// Overwrites one decision node's strategy sums (and regrets, if given) from
// blocks in the reference layout ([actions][hands]).
Status Engine::write_node(const std::vector<dcfr_step>& path, const float* regrets, const float* sums) {
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  uint32_t node = 0;
  Status s = walk(path, node, reach, to_canon);
  if (!s.ok()) return s;
  const GNode& nd = g.nodes[node];
  if (nd.kind != N_PLAYER) return bad_path("not a decision node");
  if (compressed_) return Status{DCFR_ERR_UNSUPPORTED, "write_node takes f32 storage"};
  const int q = nd.player, n = g.n[q];
  for (int a = 0; a < nd.nchild; a++) {
    if (sums)
      CK(cudaMemcpyAsync(sums_ + gpu_off_[node] + (size_t)a * hp_[q], sums + (size_t)a * n, (size_t)n * 4,
                         cudaMemcpyHostToDevice, stream_));
    if (regrets)
      CK(cudaMemcpyAsync(regrets_ + gpu_off_[node] + (size_t)a * hp_[q], regrets + (size_t)a * n, (size_t)n * 4,
                         cudaMemcpyHostToDevice, stream_));
  }
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::ensure_discounts(uint32_t max_t) {
  if (disc_table_ && max_t < disc_len_) return Status();
  uint32_t len = std::max<uint32_t>(max_t + 1, disc_len_ * 2);
  std::vector<DiscountD> tab(len);
  for (uint32_t t = 0; t < len; t++) tab[t] = discount_for(t, g.cfg.dcfr);
  CK(cudaStreamSynchronize(stream_));
  free_graphs();
  dfree(disc_table_);
  Status s;
  if (!(s = dalloc(disc_table_, len, "discounts")).ok()) return s;
  CK(cudaMemcpy(disc_table_, tab.data(), len * sizeof(DiscountD), cudaMemcpyHostToDevice));
  disc_len_ = len;
  return Status();
}

Status Engine::capture_graphs() {
  if (iter_graph_) return Status();
  const auto t0 = std::chrono::steady_clock::now();
  cudaGraph_t graph;
  // One DCFR iteration: t += 1, then player 0's and player 1's traversals
  // with the same discounts (lib.rs:577-585).
  // The first traversal's start kernel advances the iteration.
  CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  enqueue_traversal(*full_[0], M_CFR, root_rows_, nullptr, true);
  enqueue_traversal(*full_[1], M_CFR, root_rows_ + stride_, nullptr);
  CK(cudaStreamEndCapture(stream_, &graph));
  CK(cudaGraphInstantiate(&iter_graph_, graph, 0));
  cudaGraphDestroy(graph);
  iter_kernels_ = full_[0]->kernels + full_[1]->kernels;
  setup.iteration_graph_ms += ms_since(t0);
  return Status();
}

// The best-response and average-strategy traversal pairs (exploitability,
// root values), captured on their first use.
Status Engine::capture_eval_graphs() {
  if (br_graph_) return Status();
  const auto t0 = std::chrono::steady_clock::now();
  cudaGraph_t graph;
  for (int mode : {M_BR, M_AVG}) {
    CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    enqueue_traversal(*full_[0], mode, root_rows_, root_out_);
    enqueue_traversal(*full_[1], mode, root_rows_ + stride_, root_out_ + stride_);
    CK(cudaStreamEndCapture(stream_, &graph));
    CK(cudaGraphInstantiate(mode == M_BR ? &br_graph_ : &avg_graph_, graph, 0));
    cudaGraphDestroy(graph);
  }
  pair_kernels_ = full_[0]->kernels + full_[1]->kernels;
  setup.eval_graphs_ms += ms_since(t0);
  return Status();
}

// Records an event-record node into the profiled graph being captured and
// remembers it with the class of the interval it closes.
void Engine::mark(int cls) {
  if (!marking_ || !mark_status_.ok()) return;
  // An external event record becomes a graph node (a plain record inside a
  // capture only orders streams).
  cudaError_t e = cudaEventRecordWithFlags(ev0_, stream_, cudaEventRecordExternal);
  cudaStreamCaptureStatus st;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(stream_, &st, nullptr, nullptr, &deps, &ndeps);
  if (e != cudaSuccess || ndeps != 1) {
    mark_status_ = e != cudaSuccess ? cuda_status(e, "profiled graph capture") : Status{DCFR_ERR_CUDA, "profiled graph capture: unexpected dependencies"};
    return;
  }
  marking_->push_back(Mark{deps[0], cls});
}

// One DCFR iteration as in capture_graphs, with an event at the start and at
// every kernel-class boundary.
Status Engine::capture_profiled_graph() {
  if (prof_exec_) return Status();
  marks_.clear();
  mark_status_ = Status();
  marking_ = &marks_;
  CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  mark(-1);
  enqueue_traversal(*full_[0], M_CFR, root_rows_, nullptr, true);
  enqueue_traversal(*full_[1], M_CFR, root_rows_ + stride_, nullptr);
  marking_ = nullptr;
  cudaError_t e = cudaStreamEndCapture(stream_, &prof_graph_);
  if (!mark_status_.ok()) return mark_status_;
  CK(e);
  CK(cudaGraphInstantiate(&prof_exec_, prof_graph_, 0));
  return Status();
}

Status Engine::iterate_profiled(uint32_t n, dcfr_kernel_profile& out) {
  std::memset(&out, 0, sizeof out);
  Status s;
  if (!(s = ensure_discounts(iterations + n + 1)).ok()) return s;
  if (!(s = capture_graphs()).ok()) return s;
  if (!(s = capture_profiled_graph()).ok()) return s;
  const size_t M = marks_.size();
  while (prof_events_.size() < (size_t)n * M) {
    cudaEvent_t ev;
    CK(cudaEventCreate(&ev));
    prof_events_.push_back(ev);
  }
  for (uint32_t i = 0; i < n; i++) {
    for (size_t m = 0; m < M; m++)
      CK(cudaGraphExecEventRecordNodeSetEvent(prof_exec_, marks_[m].node, prof_events_[(size_t)i * M + m]));
    CK(cudaGraphLaunch(prof_exec_, stream_));
    launches += iter_kernels_;
  }
  iterations += n;
  CK(cudaStreamSynchronize(stream_));
  out.iterations = n;
  for (uint32_t i = 0; i < n; i++)
    for (size_t m = 0; m < M; m++) {
      const size_t k = (size_t)i * M + m;
      if (k == 0) continue;
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, prof_events_[k - 1], prof_events_[k]));
      // The first event of an iteration closes the gap after the previous one.
      const int cls = m == 0 ? DCFR_KERNEL_OTHER : marks_[m].cls;
      out.ms[cls] += ms;
    }
  if (n > 0) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, prof_events_[0], prof_events_[(size_t)n * M - 1]));
    out.total_ms = ms;
    last_iterate_ms = ms;
  }
  for (int c = 0; c < DCFR_KERNEL_CLASSES; c++) {
    out.launches[c] = (uint64_t)n * (full_[0]->class_kernels[c] + full_[1]->class_kernels[c]);
    out.bytes[c] = (double)n * (full_[0]->class_bytes[c] + full_[1]->class_bytes[c]);
  }
  return Status();
}

Status Engine::iterate(uint32_t n) {
  Status s;
  if (!(s = ensure_discounts(iterations + n + 1)).ok()) return s;
  if (!(s = capture_graphs()).ok()) return s;
  CK(cudaEventRecord(ev0_, stream_));
  for (uint32_t i = 0; i < n; i++) {
    CK(cudaGraphLaunch(iter_graph_, stream_));
    launches += iter_kernels_;
  }
  CK(cudaEventRecord(ev1_, stream_));
  iterations += n;
  CK(cudaEventSynchronize(ev1_));
  if (!leaf_status_.ok()) return leaf_status_;
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_iterate_ms = ms;
  return Status();
}

Status Engine::sync() {
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// root_values (cfr.rs:482-490): sum over hands of value * weight in f64.
Status Engine::mode_root_values(int mode, double out[2]) {
  Status s;
  if (!(s = capture_eval_graphs()).ok()) return s;
  CK(cudaGraphLaunch(mode == M_BR ? br_graph_ : avg_graph_, stream_));
  launches += pair_kernels_;
  std::vector<float> rows((size_t)2 * stride_);
  CK(cudaMemcpyAsync(rows.data(), root_out_, rows.size() * 4, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  for (int p = 0; p < 2; p++) {
    double acc = -0.0;
    for (int h = 0; h < g.n[p]; h++) acc += (double)rows[(size_t)p * stride_ + h] * (double)g.weights[p][h];
    out[p] = acc;
  }
  return Status();
}

// exploitability (cfr.rs:494-502).
Status Engine::exploitability(double& out) {
  double br[2];
  Status s = mode_root_values(M_BR, br);
  if (!s.ok()) return s;
  if (g.cfg.rake_rate > 0.0 && g.cfg.rake_cap > 0.0) {
    double ev[2];
    if (!(s = mode_root_values(M_AVG, ev)).ok()) return s;
    out = ((br[0] - ev[0]) + (br[1] - ev[1])) / 2.0;
  } else {
    out = (br[0] + br[1]) / 2.0;
  }
  return Status();
}

Status Engine::root_values(double out[2]) { return mode_root_values(M_AVG, out); }

// Root values of both traversals with double rows (br64.cu): best response
// (M_BR) or the average strategy (M_AVG); sum over hands of value * weight.
Status Engine::fp64_root_values(int mode, double out[2]) {
  Status s;
  if (!(s = ensure_fast_layouts()).ok()) return s;
  const size_t N = g.nodes.size();
  if (!reach64_) {
    if (!(s = dalloc(reach64_, (size_t)max_slots_ * stride_, "FP64 reach rows")).ok()) return s;
    if (!(s = dalloc(vals64_, N * (size_t)stride_, "FP64 value rows")).ok()) return s;
    if (!(s = dalloc(root_rows64_, (size_t)2 * stride_, "FP64 root rows")).ok()) return s;
    std::vector<double> rr((size_t)2 * stride_, 0.0);
    for (int p = 0; p < 2; p++)
      for (int i = 0; i < g.n[p ^ 1]; i++) rr[(size_t)p * stride_ + i] = (double)g.weights[p ^ 1][i];
    CK(cudaMemcpy(root_rows64_, rr.data(), rr.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemsetAsync(reach64_, 0, (size_t)max_slots_ * stride_ * 8, stream_));
    CK(cudaMemsetAsync(vals64_, 0, N * (size_t)stride_ * 8, stream_));
  }
  std::vector<double> row((size_t)stride_);
  for (int p = 0; p < 2; p++) {
    const Plan& plan = *full_[p];
    const int o = p ^ 1;
    CK(cudaMemsetAsync(alive_, 0, (size_t)plan.nslots * 4, stream_));
    CK(cudaMemsetAsync(alive_, 1, 4, stream_));
    CK(cudaMemcpyAsync(reach64_, root_rows64_ + (size_t)p * stride_, (size_t)stride_ * 8, cudaMemcpyDeviceToDevice,
                       stream_));
    Row64Args A;
    A.sums = sums_;
    A.sq = compressed_ ? sq_ : nullptr;
    A.sscale = sscale_;
    A.reach = reach64_;
    A.vals = vals64_;
    A.alive = alive_;
    for (int q = 0; q < 2; q++) {
      A.hc1[q] = hc1_[q];
      A.hc2[q] = hc2_[q];
      A.n[q] = g.n[q];
      A.hp[q] = hp_[q];
    }
    A.perm = perm_;
    A.chance_cards = chance_cards_;
    A.iso = iso_;
    A.stride = stride_;
    A.p = p;
    const size_t layers = std::max({plan.tree_layers.size(), plan.down.size(), plan.seg_down.size()});
    for (size_t l = 0; l < layers; l++) {
      if (l < plan.tree_layers.size() && plan.tree_layers[l].second)
        launch_fused_down64(A, plan.d_trees + plan.tree_layers[l].first, (int)plan.tree_layers[l].second,
                            plan.d_fdown, stream_);
      if (l < plan.seg_down.size())
        for (const Plan::Level& lv : plan.seg_down[l])
          if (lv.count) launch_down64(A, plan.d_down + lv.first, (int)lv.count, hp_[o], stream_);
      if (l < plan.down.size() && plan.down[l].count)
        launch_down64(A, plan.d_down + plan.down[l].first, (int)plan.down[l].count, hp_[o], stream_);
    }
    if (!plan.h_fast.empty()) {
      FastArgs64 F;
      F.reach = reach64_;
      F.vals = vals64_;
      F.alive = alive_;
      F.cat = fcat_;
      F.seg = fseg_;
      F.rec = frec_;
      F.same = same_[p];
      F.cstride = fcstride_;
      F.tstride = tstride_;
      F.emax = femax_;
      for (int q = 0; q < 2; q++) {
        F.n[q] = g.n[q];
        F.hp[q] = hp_[q];
      }
      F.stride = stride_;
      F.p = p;
      launch_warp_terminal64(F, plan.d_fast, plan.d_units, (int)plan.h_units.size(), (int)plan.h_fast.size(),
                               term_warps_[1], term_blocks_[1],
                             stream_);
    }
    for (size_t l = layers; l-- > 0;) {
      if (l < plan.up.size() && plan.up[l].count)
        launch_up64(mode, A, plan.d_up + plan.up[l].first, (int)plan.up[l].count, hp_[p], stream_);
      if (l < plan.seg_up.size())
        for (size_t d = plan.seg_up[l].size(); d-- > 0;) {
          const Plan::Level& lv = plan.seg_up[l][d];
          if (lv.count) launch_up64(mode, A, plan.d_up + lv.first, (int)lv.count, hp_[p], stream_);
        }
      if (l < plan.tree_layers.size() && plan.tree_layers[l].second)
        launch_fused_up64(mode, A, plan.d_trees + plan.tree_layers[l].first, (int)plan.tree_layers[l].second,
                          plan.d_fup, stream_);
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(row.data(), vals64_ + (size_t)plan.root * stride_, (size_t)stride_ * 8,
                       cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    double acc = 0.0;
    for (int h = 0; h < g.n[p]; h++) acc += row[h] * (double)g.weights[p][h];
    out[p] = acc;
  }
  return Status();
}

// exploitability (cfr.rs:494-502) from the FP64 traversals.
Status Engine::exploitability_fp64(double& out, double br[2]) {
  Status s = fp64_root_values(M_BR, br);
  if (!s.ok()) return s;
  if (g.cfg.rake_rate > 0.0 && g.cfg.rake_cap > 0.0) {
    double ev[2];
    if (!(s = fp64_root_values(M_AVG, ev)).ok()) return s;
    out = ((br[0] - ev[0]) + (br[1] - ev[1])) / 2.0;
  } else {
    out = (br[0] + br[1]) / 2.0;
  }
  return Status();
}

Status Engine::traverse(int p, int mode, uint32_t t, float* out) {
  if (p < 0 || p > 1 || mode < 0 || mode > 2) {
    Status s;
    s.code = DCFR_ERR_INVALID_ARG;
    s.msg = "traverse: bad player or mode";
    return s;
  }
  DiscountD d = discount_for(t, g.cfg.dcfr);
  CK(cudaMemcpyAsync(cur_disc_, &d, sizeof d, cudaMemcpyHostToDevice, stream_));
  enqueue_traversal(*full_[p], mode, root_rows_ + (size_t)p * stride_, root_out_ + (size_t)p * stride_);
  launches += full_[p]->kernels;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, root_out_ + (size_t)p * stride_, (size_t)g.n[p] * 4, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// dcfr_solve with its device time: CUDA events on the handle's stream at
// the start and at the end (iterations, checks and any first-use graph
// capture between them).
Status Engine::solve(const dcfr_solve_options& opts, const volatile int32_t* cancel, dcfr_progress_cb cb, void* user,
                     dcfr_progress& progress) {
  CK(cudaEventRecord(ev0_, stream_));
  Status s = solve_loop(opts, cancel, cb, user, progress);
  if (!s.ok()) return s;
  CK(cudaEventRecord(ev1_, stream_));
  CK(cudaEventSynchronize(ev1_));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_solve_ms = ms;
  return Status();
}

Status Engine::solve_loop(const dcfr_solve_options& opts, const volatile int32_t* cancel, dcfr_progress_cb cb,
                          void* user, dcfr_progress& progress) {
  const double pot = (double)g.cfg.root.pot;
  const uint32_t check_every = std::max(opts.check_every, 1u);
  progress.iteration = iterations;
  progress.max_iterations = opts.max_iterations;
  progress.exploitability = last_exploitability;
  progress.exploitability_pct = 100.0 * last_exploitability / pot;
  progress.finished = 0;
  const double target = opts.target_exploitability_pct * pot / 100.0;
  uint32_t next_check = iterations + check_every;
  bool has_last = false;
  uint32_t last_t = 0;
  double last_e = 0.0;
  Status s;
  if (!(s = ensure_discounts(opts.max_iterations + 1)).ok()) return s;
  if (!(s = capture_graphs()).ok()) return s;
  while (iterations < opts.max_iterations) {
    if (cancel && *cancel) {
      progress.finished = 1;
      CK(cudaStreamSynchronize(stream_));
      return Status();
    }
    iterations += 1;
    CK(cudaGraphLaunch(iter_graph_, stream_));
    launches += iter_kernels_;
    bool last = iterations >= opts.max_iterations;
    if (iterations >= next_check || last) {
      double e;
      if (!(s = exploitability(e)).ok()) return s;
      last_exploitability = e;
      progress.iteration = iterations;
      progress.exploitability = e;
      progress.exploitability_pct = 100.0 * e / pot;
      bool done = progress.exploitability_pct <= opts.target_exploitability_pct || last;
      progress.finished = done ? 1 : 0;
      bool keep = cb ? cb(&progress, user) != 0 : true;
      if (done || !keep) {
        progress.finished = 1;
        return Status();
      }
      uint32_t t = iterations;
      next_check = t + next_gap(has_last, last_t, last_e, t, e, target, check_every);
      has_last = true;
      last_t = t;
      last_e = e;
    }
  }
  progress.finished = 1;
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::download(float* regrets, float* sums) {
  if (!compressed_) {
    // Packed on the device and copied straight into the caller's arrays.
    Status s;
    if (regrets && !(s = storage_out(regrets_, regrets, 4)).ok()) return s;
    if (sums && !(s = storage_out(sums_, sums, 4)).ok()) return s;
    return Status();
  }
  // Decoded as load_regrets / load_strat do (storage.rs:226-268).
  std::vector<float> r(gpu_len_), sm(gpu_len_);
  std::vector<int16_t> rq(gpu_len_);
  std::vector<uint16_t> sq(gpu_len_);
  std::vector<float> rs, ss;
  Status s = download_compressed_raw(rq, sq, rs, ss);
  if (!s.ok()) return s;
  for (uint32_t v = 0; v < g.nodes.size(); v++) {
    const GNode& nd = g.nodes[v];
    if (nd.kind != N_PLAYER) continue;
    const size_t len = (size_t)nd.nchild * hp_[nd.player];
    const float rsc = rs[nd.index] / 32767.0f, ssc = ss[nd.index] / 65535.0f;
    for (size_t i = 0; i < len; i++) {
      r[gpu_off_[v] + i] = (float)rq[gpu_off_[v] + i] * rsc;
      sm[gpu_off_[v] + i] = (float)sq[gpu_off_[v] + i] * ssc;
    }
  }
  for (uint32_t v = 0; v < g.nodes.size(); v++) {
    const GNode& nd = g.nodes[v];
    if (nd.kind != N_PLAYER) continue;
    int q = nd.player, n = g.n[q];
    for (int a = 0; a < nd.nchild; a++) {
      if (regrets)
        std::memcpy(regrets + nd.ref_offset + (size_t)a * n, r.data() + gpu_off_[v] + (size_t)a * hp_[q], n * 4);
      if (sums) std::memcpy(sums + nd.ref_offset + (size_t)a * n, sm.data() + gpu_off_[v] + (size_t)a * hp_[q], n * 4);
    }
  }
  return Status();
}

// Decision nodes in the reference's storage order (the device blocks are in
// the same order, gpu_off_ increasing), cut into chunks of whole nodes of at
// most STAGE_MAX elements; built on the first transfer.
Status Engine::storage_chunks() {
  if (!schunks_.empty() || g.storage_len == 0) return Status();
  constexpr uint64_t STAGE_MAX = (uint64_t)1 << 26;
  const std::vector<uint32_t> players = players_in_storage_order(g);
  std::vector<StorageBlockD> blk(players.size());
  std::vector<StorageChunk> chunks;
  StorageChunk c{0, 0, 0, 0};
  uint64_t stage = 0;
  for (size_t i = 0; i < players.size(); i++) {
    const GNode& nd = g.nodes[players[i]];
    const int q = nd.player;
    const uint64_t len = (uint64_t)nd.nchild * (uint64_t)g.n[q];
    if (c.count > 0 && c.len + len > STAGE_MAX) {
      chunks.push_back(c);
      c = StorageChunk{(uint32_t)i, 0, nd.ref_offset, 0};
    }
    if (c.count == 0) c = StorageChunk{(uint32_t)i, 0, nd.ref_offset, 0};
    blk[i] = StorageBlockD{gpu_off_[players[i]], nd.ref_offset - c.host, nd.nchild, (uint32_t)g.n[q],
                           (uint32_t)hp_[q], 0};
    c.count++;
    c.len += len;
    stage = std::max(stage, c.len);
  }
  if (c.count > 0) chunks.push_back(c);
  Status s;
  if (!(s = dalloc(sblk_, blk.size(), "storage transfer table")).ok()) return s;
  CK(cudaMemcpy(sblk_, blk.data(), blk.size() * sizeof(StorageBlockD), cudaMemcpyHostToDevice));
  stage_len_ = stage;
  schunks_ = std::move(chunks);
  return Status();
}

namespace {
// A device staging buffer freed on every return path.
struct Staging {
  void* p = nullptr;
  ~Staging() {
    if (p) cudaFree(p);
  }
};
}  // namespace

// Device storage (elements of elem_bytes) to the caller's reference-layout
// array: per chunk, one pack launch and one copy to host memory.
Status Engine::storage_out(const void* dev, void* host, int elem_bytes) {
  Status s = storage_chunks();
  if (!s.ok() || schunks_.empty()) return s;
  Staging st;
  CK(cudaMalloc(&st.p, stage_len_ * (uint64_t)elem_bytes));
  for (const StorageChunk& c : schunks_) {
    launch_storage_pack(elem_bytes, dev, st.p, sblk_ + c.first, (int)c.count, stream_);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(static_cast<char*>(host) + c.host * elem_bytes, st.p, c.len * elem_bytes,
                       cudaMemcpyDeviceToHost, stream_));
  }
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// The caller's reference-layout array to the device storage (padding
// entries zeroed): per chunk, one copy from host memory and one unpack launch.
Status Engine::storage_in(void* dev, const void* host, int elem_bytes) {
  Status s = storage_chunks();
  if (!s.ok() || schunks_.empty()) return s;
  Staging st;
  CK(cudaMalloc(&st.p, stage_len_ * (uint64_t)elem_bytes));
  for (const StorageChunk& c : schunks_) {
    CK(cudaMemcpyAsync(st.p, static_cast<const char*>(host) + c.host * elem_bytes, c.len * elem_bytes,
                       cudaMemcpyHostToDevice, stream_));
    launch_storage_unpack(elem_bytes, dev, st.p, sblk_ + c.first, (int)c.count, stream_);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::download_compressed_raw(std::vector<int16_t>& rq, std::vector<uint16_t>& sq, std::vector<float>& rs,
                                       std::vector<float>& ss) {
  const size_t slots = std::max<size_t>(g.player_nodes, 1);
  rq.resize(gpu_len_);
  sq.resize(gpu_len_);
  rs.resize(slots);
  ss.resize(slots);
  CK(cudaMemcpyAsync(rq.data(), rq_, gpu_len_ * 2, cudaMemcpyDeviceToHost, stream_));
  CK(cudaMemcpyAsync(sq.data(), sq_, gpu_len_ * 2, cudaMemcpyDeviceToHost, stream_));
  CK(cudaMemcpyAsync(rs.data(), rscale_, slots * 4, cudaMemcpyDeviceToHost, stream_));
  CK(cudaMemcpyAsync(ss.data(), sscale_, slots * 4, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::download_compressed(int16_t* regrets, uint16_t* sums, float* rscale, float* sscale) {
  if (!compressed_) return Status{DCFR_ERR_UNSUPPORTED, "the solver's storage is f32"};
  Status s;
  if (regrets && !(s = storage_out(rq_, regrets, 2)).ok()) return s;
  if (sums && !(s = storage_out(sq_, sums, 2)).ok()) return s;
  if (g.player_nodes) {
    if (rscale) CK(cudaMemcpyAsync(rscale, rscale_, (size_t)g.player_nodes * 4, cudaMemcpyDeviceToHost, stream_));
    if (sscale) CK(cudaMemcpyAsync(sscale, sscale_, (size_t)g.player_nodes * 4, cudaMemcpyDeviceToHost, stream_));
  }
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::upload_compressed(const int16_t* regrets, const uint16_t* sums, const float* rscale,
                                 const float* sscale) {
  if (!compressed_) return Status{DCFR_ERR_UNSUPPORTED, "the solver's storage is f32"};
  Status s;
  if (!(s = storage_in(rq_, regrets, 2)).ok()) return s;
  if (!(s = storage_in(sq_, sums, 2)).ok()) return s;
  if (g.player_nodes) {
    CK(cudaMemcpyAsync(rscale_, rscale, (size_t)g.player_nodes * 4, cudaMemcpyHostToDevice, stream_));
    CK(cudaMemcpyAsync(sscale_, sscale, (size_t)g.player_nodes * 4, cudaMemcpyHostToDevice, stream_));
  }
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

Status Engine::upload(const float* regrets, const float* sums) {
  if (compressed_) return Status{DCFR_ERR_UNSUPPORTED, "compressed storage: use dcfr_upload_storage_compressed"};
  Status s;
  if (!(s = storage_in(regrets_, regrets, 4)).ok()) return s;
  return storage_in(sums_, sums, 4);
}

Status Engine::set_iterations(uint32_t t) {
  iterations = t;
  CK(cudaMemcpyAsync(counter_, &iterations, 4, cudaMemcpyHostToDevice, stream_));
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// Average strategy of a node (lib.rs:735-743) from the device sums.
Status Engine::avg_strategy(uint32_t node, std::vector<float>& s) {
  const GNode& nd = g.nodes[node];
  int q = nd.player, n = g.n[q];
  std::vector<float> blk((size_t)nd.nchild * hp_[q]);
  if (compressed_) {
    std::vector<uint16_t> q16(blk.size());
    float sc = 0.0f;
    CK(cudaMemcpyAsync(q16.data(), sq_ + gpu_off_[node], q16.size() * 2, cudaMemcpyDeviceToHost, stream_));
    CK(cudaMemcpyAsync(&sc, sscale_ + nd.index, 4, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
    const float dec = sc / 65535.0f;
    for (size_t i = 0; i < blk.size(); i++) blk[i] = (float)q16[i] * dec;
  } else {
    CK(cudaMemcpyAsync(blk.data(), sums_ + gpu_off_[node], blk.size() * 4, cudaMemcpyDeviceToHost, stream_));
    CK(cudaStreamSynchronize(stream_));
  }
  s.assign((size_t)nd.nchild * n, 0.0f);
  for (int a = 0; a < nd.nchild; a++)
    std::memcpy(s.data() + (size_t)a * n, blk.data() + (size_t)a * hp_[q], n * 4);
  normalize_rows(s.data(), nd.nchild, n);
  return Status();
}

static Status bad_path(const std::string& m) {
  Status s;
  s.code = DCFR_ERR_BAD_PATH;
  s.msg = "bad path: " + m;
  return s;
}

static const char* RANKC = "23456789TJQKA";
static const char* SUITC = "cdhs";
static std::string card_name(int c) { return std::string(1, RANKC[c >> 2]) + SUITC[c & 3]; }

// walk (lib.rs:746-825).
Status Engine::walk(const std::vector<dcfr_step>& path, uint32_t& node, std::vector<float> reach[2],
                    std::vector<uint32_t> to_canon[2]) {
  static const uint8_t PAIRS[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  uint32_t id = 0;
  for (int x = 0; x < 2; x++) {
    reach[x] = g.weights[x];
    to_canon[x].resize(g.n[x]);
    for (int i = 0; i < g.n[x]; i++) to_canon[x][i] = (uint32_t)i;
  }
  int suit_map[4] = {0, 1, 2, 3};
  for (size_t depth = 0; depth < path.size(); depth++) {
    const dcfr_step& st = path[depth];
    const GNode nd = g.nodes[id];
    if (nd.kind == N_PLAYER && st.kind == 0) {
      auto acts = g.actions(id);
      Act a{st.action_kind, st.action_kind == DCFR_RAISE ? st.amount : 0};
      size_t ai = std::find(acts.begin(), acts.end(), a) - acts.begin();
      if (ai == acts.size()) return bad_path("action not available at depth " + std::to_string(depth));
      int q = nd.player, n = g.n[q];
      std::vector<float> s;
      Status ss = avg_strategy(id, s);
      if (!ss.ok()) return ss;
      for (int i = 0; i < n; i++) reach[q][i] *= s[ai * n + i];
      id = nd.first + (uint32_t)ai;
    } else if (nd.kind == N_CHANCE && st.kind == 1) {
      int c = st.card;
      if (c < 0 || c >= 52) return bad_path("card id out of range at depth " + std::to_string(depth));
      int cc = (c >> 2) * 4 + suit_map[c & 3];
      int canonical = -1;
      for (uint32_t ch = nd.first; ch < nd.first + nd.nchild; ch++)
        if (g.nodes[ch].card == cc) {
          id = ch;
          canonical = cc;
          break;
        }
      if (canonical < 0) {
        const ChanceIso& info = g.chance[nd.index];
        size_t j = std::find(info.cards.begin(), info.cards.end(), (uint8_t)cc) - info.cards.begin();
        if (j == info.cards.size())
          return bad_path("card " + card_name(c) + " not in the tree at depth " + std::to_string(depth));
        int ci = info.ci[j], pair = info.pair[j];
        int a = PAIRS[pair][0], b = PAIRS[pair][1];
        for (int& sm : suit_map) sm = sm == a ? b : sm == b ? a : sm;
        for (int x = 0; x < 2; x++) {
          const auto& perm = g.perm[x][pair];
          std::vector<float> r2(reach[x].size(), 0.0f);
          for (size_t h = 0; h < reach[x].size(); h++) r2[perm[h]] = reach[x][h];
          reach[x] = r2;
          for (auto& t : to_canon[x]) t = perm[t];
        }
        id = nd.first + (uint32_t)ci;
        canonical = g.nodes[id].card;
      }
      for (int x = 0; x < 2; x++)
        for (uint32_t k : g.blocked[x][canonical]) reach[x][k] = 0.0f;
    } else {
      return bad_path("step doesn't match node kind at depth " + std::to_string(depth));
    }
  }
  node = id;
  return Status();
}

Status Engine::actions_at(const std::vector<dcfr_step>& path, std::vector<Act>& out, bool& decision) {
  uint32_t node;
  std::vector<float> reach[2];
  std::vector<uint32_t> tc[2];
  Status s = walk(path, node, reach, tc);
  if (!s.ok()) return s;
  decision = g.nodes[node].kind == N_PLAYER;
  out.clear();
  if (decision) out = g.actions(node);
  return Status();
}

// Values of traverser p at the subtree `root` under the opponent reach
// (cfr::traverse in Average mode from an interior node).
Status Engine::subtree_values(uint32_t root, int p, const std::vector<float>& opp_reach, std::vector<float>& out) {
  out.assign(g.n[p], 0.0f);
  bool any = false;
  for (float x : opp_reach) any |= x != 0.0f;
  if (!any) return Status();
  Plan plan;
  Status s;
  if (!(s = build_plan(root, p, plan)).ok()) return s;
  for (const Plan::Wave& w : plan.waves)
    if (!fast_ && ((int)w.count > wave_tasks_ || (int)w.groups > wave_groups_)) {
      s.code = DCFR_ERR_INVALID_ARG;
      s.msg = "subtree plan exceeds the terminal scratch";
      return s;
    }
  if (plan.nslots > max_slots_) {
    s.code = DCFR_ERR_INVALID_ARG;
    s.msg = "subtree plan exceeds the reach buffer";
    return s;
  }
  if (!(s = upload_plan(plan)).ok()) return s;
  std::vector<float> row(stride_, 0.0f);
  std::copy(opp_reach.begin(), opp_reach.end(), row.begin());
  float* d_row = root_out_ + (size_t)(p ^ 1) * stride_;  // scratch row
  CK(cudaMemcpyAsync(d_row, row.data(), stride_ * 4, cudaMemcpyHostToDevice, stream_));
  enqueue_traversal(plan, M_AVG, d_row, nullptr);
  launches += plan.kernels;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out.data(), vals_ + (size_t)root * stride_, (size_t)g.n[p] * 4, cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  return Status();
}

// The root's children's values for traverser q under the average strategy:
// at the root the opponent's reach is its range (as walk() gives there), so
// one traversal of the full plan (the one the solve runs, in average mode)
// leaves every child's values in its value row, with the same per-node
// arithmetic as a subtree plan from that child (subtree_values) and without
// building one plan per child. A terminal child is the exception: evaluated
// from itself (as the reference's query does) it is the traversal's root and
// takes the scalar evaluator, while below a river decision in the full tree
// it takes the batched one (cfr.rs:282-284), so it keeps its own plan.
Status Engine::root_child_values(int q, const std::vector<float>& opp_reach, std::vector<std::vector<float>>& child) {
  const GNode& nd = g.nodes[0];
  for (uint32_t a = 0; a < nd.nchild; a++) child[a].assign(g.n[q], 0.0f);
  enqueue_traversal(*full_[q], M_AVG, root_rows_ + (size_t)q * stride_, nullptr);
  launches += full_[q]->kernels;
  CK(cudaGetLastError());
  for (uint32_t a = 0; a < nd.nchild; a++)
    CK(cudaMemcpyAsync(child[a].data(), vals_ + (size_t)(nd.first + a) * stride_, (size_t)g.n[q] * 4,
                       cudaMemcpyDeviceToHost, stream_));
  CK(cudaStreamSynchronize(stream_));
  for (uint32_t a = 0; a < nd.nchild; a++) {
    const int kind = g.nodes[nd.first + a].kind;
    if (kind == N_FOLD || kind == N_SHOWDOWN) {
      Status s = subtree_values(nd.first + a, q, opp_reach, child[a]);
      if (!s.ok()) return s;
    }
  }
  return Status();
}

// query (lib.rs:842-899).
Status Engine::query(const std::vector<dcfr_step>& path, dcfr_node_info& info, std::vector<Act>& actions,
                     std::vector<uint16_t>& combos, std::vector<float>& strategy, std::vector<float>& ev,
                     std::vector<float>& reach_real) {
  uint32_t node;
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  Status s = walk(path, node, reach, to_canon);
  if (!s.ok()) return s;
  const GNode nd = g.nodes[node];
  if (nd.kind != N_PLAYER) return bad_path("not a decision node");
  const int q = nd.player, o = q ^ 1, n = g.n[q], na = nd.nchild;
  // compatible_reach (hands.rs:102-125).
  std::vector<double> compat(n);
  {
    double total = 0.0, minus[52] = {0};
    for (int k = 0; k < g.n[o]; k++) {
      float w = reach[o][k];
      if (w != 0.0f) {
        total += (double)w;
        minus[g.c1[o][k]] += (double)w;
        minus[g.c2[o][k]] += (double)w;
      }
    }
    for (int i = 0; i < n; i++) {
      double sw = g.same[q][i] == NO ? 0.0 : (double)reach[o][g.same[q][i]];
      double v = total - minus[g.c1[q][i]] - minus[g.c2[q][i]] + sw;
      compat[i] = v > 0.0 ? v : 0.0;
    }
  }
  std::vector<std::vector<float>> child(na);
  if (node == 0) {
    if (!(s = root_child_values(q, reach[o], child)).ok()) return s;
  } else {
    for (int a = 0; a < na; a++)
      if (!(s = subtree_values(nd.first + a, q, reach[o], child[a])).ok()) return s;
  }
  const double offset = g.half_pot + (double)nd.invest[q];
  std::vector<float> strat_c;
  if (!(s = avg_strategy(node, strat_c)).ok()) return s;
  ev.assign((size_t)na * n, 0.0f);
  strategy.assign((size_t)na * n, 0.0f);
  reach_real.assign(n, 0.0f);
  for (int h = 0; h < n; h++) {
    uint32_t hc = to_canon[q][h];
    reach_real[h] = reach[q][hc];
    double denom = compat[hc] * g.norm;
    for (int a = 0; a < na; a++) {
      strategy[(size_t)a * n + h] = strat_c[(size_t)a * n + hc];
      ev[(size_t)a * n + h] = denom > 0.0 ? (float)((double)child[a][hc] / denom + offset) : 0.0f;
    }
  }
  for (int p = 0; p < 2; p++) {
    double root = -0.0, now = -0.0;
    for (float x : g.weights[p]) root += (double)x;
    for (float x : reach[p]) now += (double)x;
    info.reach_fraction[p] = root > 0.0 ? now / root : 0.0;
  }
  info.player = q;
  info.num_actions = na;
  info.num_hands = n;
  info.pot = g.cfg.root.pot + (int64_t)nd.invest[0] + (int64_t)nd.invest[1];
  info.invest[0] = nd.invest[0];
  info.invest[1] = nd.invest[1];
  actions = g.actions(node);
  combos = g.combos[q];
  return Status();
}

// ranges_after (lib.rs:903-912).
Status Engine::ranges_after(const std::vector<dcfr_step>& path, float out[2][DCFR_NUM_COMBOS]) {
  uint32_t node;
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  Status s = walk(path, node, reach, to_canon);
  if (!s.ok()) return s;
  for (int p = 0; p < 2; p++) {
    for (int c = 0; c < DCFR_NUM_COMBOS; c++) out[p][c] = 0.0f;
    for (int h = 0; h < g.n[p]; h++) out[p][g.combos[p][h]] = reach[p][to_canon[p][h]];
  }
  return Status();
}

}  // namespace dcfr
