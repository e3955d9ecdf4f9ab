// C ABI of libdcfr (include/dcfr.h) over the device engine.
#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>

#include "../../include/dcfr.h"
#include "batch.hpp"
#include "engine.hpp"

struct dcfr_solver {
  std::unique_ptr<dcfr::Engine> e;
};

struct dcfr_batch {
  std::unique_ptr<dcfr::Batch> b;
};

static thread_local std::string g_error;

static int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

namespace dcfr {
// Lets the library's other translation units report through dcfr_last_error.
void set_last_error(const std::string& msg) { g_error = msg; }
}  // namespace dcfr

static int done(const dcfr::Status& s) {
  if (s.ok()) {
    g_error.clear();
    return DCFR_OK;
  }
  return fail(s.code, s.msg);
}

#define GUARD_BEGIN try {
#define GUARD_END                                                     \
  }                                                                   \
  catch (const std::bad_alloc&) {                                     \
    return fail(DCFR_ERR_OUT_OF_MEMORY, "host allocation failed");    \
  }                                                                   \
  catch (const std::exception& ex) {                                  \
    return fail(DCFR_ERR_INVALID_ARG, ex.what());                     \
  }

static std::vector<dcfr_step> steps(const dcfr_step* path, size_t n) {
  return path ? std::vector<dcfr_step>(path, path + n) : std::vector<dcfr_step>();
}

static void set_sizes(dcfr_street_sizes& s, std::initializer_list<double> bet_pot, double raise_mult) {
  std::memset(&s, 0, sizeof s);
  for (double b : bet_pot) s.bet[s.n_bet++] = dcfr_bet_size{DCFR_SIZE_POT, 0, b};
  s.raise[s.n_raise++] = dcfr_bet_size{DCFR_SIZE_MULT, 0, raise_mult};
}

extern "C" {

const char* dcfr_last_error(void) { return g_error.c_str(); }

int dcfr_config_init(dcfr_config* cfg) {
  if (!cfg) return fail(DCFR_ERR_INVALID_ARG, "cfg is NULL");
  std::memset(cfg, 0, sizeof *cfg);
  set_sizes(cfg->menu.flop, {0.33, 0.75}, 3.0);
  set_sizes(cfg->menu.turn, {0.5, 1.0}, 3.0);
  set_sizes(cfg->menu.river, {0.5, 1.0}, 3.0);
  cfg->menu.max_raises = 3;
  cfg->menu.add_allin_threshold = 1.5;
  cfg->menu.force_allin_threshold = 0.15;
  cfg->menu.merge_threshold = 0.1;
  cfg->big_blind = 100;
  cfg->max_memory_bytes = 8ull << 30;
  cfg->storage = DCFR_STORAGE_AUTO;
  cfg->isomorphism = 1;
  cfg->dcfr.alpha = 1.5;
  cfg->dcfr.beta = 0.0;
  cfg->dcfr.gamma = 3.0;
  cfg->dcfr.restart_average = 1;
  cfg->dcfr.unweighted_average = 1;
  cfg->precision = DCFR_PRECISION_FAST;
  return DCFR_OK;
}

int dcfr_estimate(const dcfr_config* cfg, dcfr_tree_stats* out) {
  if (!cfg || !out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  dcfr::Game g;
  std::string msg;
  int rc = dcfr::build_game(*cfg, g, msg, false);
  if (rc) return fail(rc, msg);
  out->player_nodes = g.stats.player;
  out->chance_nodes = g.stats.chance;
  out->terminal_nodes = g.stats.terminal;
  out->storage_cells = g.stats.cells;
  out->compressed = g.compressed ? 1 : 0;
  out->memory_bytes = dcfr::reference_memory_bytes(g.stats, g.compressed);
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_create(const dcfr_config* cfg, dcfr_solver** out) {
  if (!cfg || !out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  GUARD_BEGIN
  std::unique_ptr<dcfr::Engine> e;
  dcfr::Status s = dcfr::Engine::create(*cfg, e);
  if (!s.ok()) return done(s);
  dcfr_solver* h = new dcfr_solver();
  h->e = std::move(e);
  *out = h;
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

void dcfr_destroy(dcfr_solver* s) { delete s; }

#define NEED(h)                                                       \
  if (!(h) || !(h)->e) return fail(DCFR_ERR_INVALID_ARG, "NULL solver")

int dcfr_solve(dcfr_solver* s, const dcfr_solve_options* opts, const volatile int32_t* cancel, dcfr_progress_cb cb,
               void* user, dcfr_progress* out) {
  NEED(s);
  if (!opts || !out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  return done(s->e->solve(*opts, cancel, cb, user, *out));
  GUARD_END
}

int dcfr_iterate(dcfr_solver* s, uint32_t n) {
  NEED(s);
  GUARD_BEGIN
  return done(s->e->iterate(n));
  GUARD_END
}

int dcfr_synchronize(dcfr_solver* s) {
  NEED(s);
  return done(s->e->sync());
}

int dcfr_exploitability(dcfr_solver* s, double* out) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  return done(s->e->exploitability(*out));
  GUARD_END
}

int dcfr_exploitability_fp64(dcfr_solver* s, double* out, double best_response[2]) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  double br[2] = {0.0, 0.0};
  dcfr::Status st = s->e->exploitability_fp64(*out, br);
  if (st.ok() && best_response) {
    best_response[0] = br[0];
    best_response[1] = br[1];
  }
  return done(st);
  GUARD_END
}

int dcfr_create_depth_limited(const dcfr_config* cfg, dcfr_mlp* net, dcfr_solver** out) {
  if (!cfg || !out || !net) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  GUARD_BEGIN
  std::unique_ptr<dcfr::Engine> e;
  dcfr::Status st = dcfr::Engine::create_depth_limited(*cfg, net, DCFR_TURN, e);
  if (!st.ok()) return done(st);
  *out = new dcfr_solver{std::move(e)};
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_node_storage(dcfr_solver* s, const dcfr_step* path, size_t n, uint64_t* offset, int32_t* num_actions,
                      int32_t* num_hands) {
  NEED(s);
  if (!offset || !num_actions || !num_hands) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  int na = 0, nh = 0;
  dcfr::Status st = s->e->node_storage(steps(path, n), *offset, na, nh);
  *num_actions = na;
  *num_hands = nh;
  return done(st);
  GUARD_END
}

int dcfr_write_node(dcfr_solver* s, const dcfr_step* path, size_t n, const float* regrets, const float* sums) {
  NEED(s);
  if (!regrets && !sums) return fail(DCFR_ERR_INVALID_ARG, "nothing to write");
  GUARD_BEGIN
  return done(s->e->write_node(steps(path, n), regrets, sums));
  GUARD_END
}

int dcfr_root_values(dcfr_solver* s, double out[2]) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  GUARD_BEGIN
  return done(s->e->root_values(out));
  GUARD_END
}

int dcfr_iterations(const dcfr_solver* s, uint32_t* out) {
  NEED(s);
  *out = s->e->iterations;
  return DCFR_OK;
}

int dcfr_last_exploitability(const dcfr_solver* s, double* out) {
  NEED(s);
  *out = s->e->last_exploitability;
  return DCFR_OK;
}

int dcfr_stats(const dcfr_solver* s, dcfr_tree_stats* out) {
  NEED(s);
  const dcfr::Game& g = s->e->g;
  out->player_nodes = g.stats.player;
  out->chance_nodes = g.stats.chance;
  out->terminal_nodes = g.stats.terminal;
  out->storage_cells = g.stats.cells;
  out->compressed = g.compressed ? 1 : 0;
  out->memory_bytes = dcfr::reference_memory_bytes(g.stats, g.compressed);
  return DCFR_OK;
}

int dcfr_isomorphic_pairs(const dcfr_solver* s, int32_t* out) {
  NEED(s);
  *out = s->e->isomorphic_pairs();
  return DCFR_OK;
}

int dcfr_hands(const dcfr_solver* s, int32_t p, uint16_t* combos, float* weights, int32_t* n) {
  NEED(s);
  if (p < 0 || p > 1 || !n) return fail(DCFR_ERR_INVALID_ARG, "bad player");
  const dcfr::Game& g = s->e->g;
  *n = g.n[p];
  if (combos) std::memcpy(combos, g.combos[p].data(), g.n[p] * 2);
  if (weights) std::memcpy(weights, g.weights[p].data(), g.n[p] * 4);
  return DCFR_OK;
}

int dcfr_is_decision(dcfr_solver* s, const dcfr_step* path, size_t n, int32_t* out) {
  NEED(s);
  GUARD_BEGIN
  std::vector<dcfr::Act> acts;
  bool dec = false;
  dcfr::Status st = s->e->actions_at(steps(path, n), acts, dec);
  *out = st.ok() && dec ? 1 : 0;
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_actions_at(dcfr_solver* s, const dcfr_step* path, size_t n, dcfr_action* actions, size_t cap,
                    size_t* count) {
  NEED(s);
  GUARD_BEGIN
  std::vector<dcfr::Act> acts;
  bool dec = false;
  dcfr::Status st = s->e->actions_at(steps(path, n), acts, dec);
  if (!st.ok()) return done(st);
  if (count) *count = acts.size();
  for (size_t i = 0; i < acts.size() && i < cap && actions; i++) actions[i] = dcfr_action{acts[i].kind, 0, acts[i].amount};
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_query_sizes(dcfr_solver* s, const dcfr_step* path, size_t n, int32_t* num_actions, int32_t* num_hands) {
  NEED(s);
  GUARD_BEGIN
  std::vector<dcfr::Act> acts;
  bool dec = false;
  dcfr::Status st = s->e->actions_at(steps(path, n), acts, dec);
  if (!st.ok()) return done(st);
  if (!dec) return fail(DCFR_ERR_BAD_PATH, "bad path: not a decision node");
  // The acting player of the node reached by the path.
  uint32_t node = 0;
  {
    // Re-walk cheaply through actions_at's node: the decision's player is
    // read from the tree by following the same steps.
    const dcfr::Game& g = s->e->g;
    for (size_t i = 0; i < n; i++) {
      const dcfr::GNode& nd = g.nodes[node];
      if (nd.kind == dcfr::N_PLAYER) {
        auto a = g.actions(node);
        dcfr::Act want{path[i].action_kind, path[i].action_kind == DCFR_RAISE ? path[i].amount : 0};
        node = nd.first + (uint32_t)(std::find(a.begin(), a.end(), want) - a.begin());
      } else {
        // Chance: any child has the same acting player at its root.
        node = nd.first;
      }
    }
  }
  int q = s->e->g.nodes[node].player;
  if (num_actions) *num_actions = (int32_t)acts.size();
  if (num_hands) *num_hands = s->e->g.n[q];
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_query(dcfr_solver* s, const dcfr_step* path, size_t n, dcfr_node_info* info, dcfr_action* actions,
               uint16_t* combos, float* strategy, float* ev, float* reach) {
  NEED(s);
  if (!info) return fail(DCFR_ERR_INVALID_ARG, "NULL info");
  GUARD_BEGIN
  std::vector<dcfr::Act> acts;
  std::vector<uint16_t> cb;
  std::vector<float> st, e, r;
  dcfr::Status ss = s->e->query(steps(path, n), *info, acts, cb, st, e, r);
  if (!ss.ok()) return done(ss);
  if (actions)
    for (size_t i = 0; i < acts.size(); i++) actions[i] = dcfr_action{acts[i].kind, 0, acts[i].amount};
  if (combos) std::memcpy(combos, cb.data(), cb.size() * 2);
  if (strategy) std::memcpy(strategy, st.data(), st.size() * 4);
  if (ev) std::memcpy(ev, e.data(), e.size() * 4);
  if (reach) std::memcpy(reach, r.data(), r.size() * 4);
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

int dcfr_ranges_after(dcfr_solver* s, const dcfr_step* path, size_t n, float out[2][DCFR_NUM_COMBOS]) {
  NEED(s);
  GUARD_BEGIN
  return done(s->e->ranges_after(steps(path, n), out));
  GUARD_END
}

int dcfr_storage_len(const dcfr_solver* s, uint64_t* len) {
  NEED(s);
  *len = s->e->g.storage_len;
  return DCFR_OK;
}

int dcfr_download_storage(dcfr_solver* s, float* regrets, float* sums, uint64_t len) {
  NEED(s);
  if (len != s->e->g.storage_len) return fail(DCFR_ERR_INVALID_ARG, "storage length mismatch");
  GUARD_BEGIN
  return done(s->e->download(regrets, sums));
  GUARD_END
}

int dcfr_upload_storage(dcfr_solver* s, const float* regrets, const float* sums, uint64_t len) {
  NEED(s);
  if (len != s->e->g.storage_len || !regrets || !sums) return fail(DCFR_ERR_INVALID_ARG, "storage length mismatch");
  GUARD_BEGIN
  return done(s->e->upload(regrets, sums));
  GUARD_END
}

int dcfr_storage_slots(const dcfr_solver* s, uint64_t* slots) {
  NEED(s);
  if (!slots) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *slots = s->e->slots();
  return DCFR_OK;
}

int dcfr_download_storage_compressed(dcfr_solver* s, int16_t* regrets, uint16_t* sums, float* regret_scale,
                                     float* sum_scale, uint64_t len, uint64_t slots) {
  NEED(s);
  if (len != s->e->g.storage_len || slots != s->e->slots())
    return fail(DCFR_ERR_INVALID_ARG, "storage length or slot count mismatch");
  GUARD_BEGIN
  return done(s->e->download_compressed(regrets, sums, regret_scale, sum_scale));
  GUARD_END
}

int dcfr_upload_storage_compressed(dcfr_solver* s, const int16_t* regrets, const uint16_t* sums,
                                   const float* regret_scale, const float* sum_scale, uint64_t len, uint64_t slots) {
  NEED(s);
  if (len != s->e->g.storage_len || slots != s->e->slots() || !regrets || !sums || !regret_scale || !sum_scale)
    return fail(DCFR_ERR_INVALID_ARG, "storage length or slot count mismatch");
  GUARD_BEGIN
  return done(s->e->upload_compressed(regrets, sums, regret_scale, sum_scale));
  GUARD_END
}

int dcfr_set_iterations(dcfr_solver* s, uint32_t t) {
  NEED(s);
  return done(s->e->set_iterations(t));
}

int dcfr_traverse(dcfr_solver* s, int32_t p, int32_t mode, uint32_t t, float* out) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "NULL out");
  GUARD_BEGIN
  return done(s->e->traverse(p, mode, t, out));
  GUARD_END
}

int dcfr_kernel_launches(const dcfr_solver* s, uint64_t* out) {
  NEED(s);
  *out = s->e->launches;
  return DCFR_OK;
}

int dcfr_last_iterate_ms(dcfr_solver* s, double* ms) {
  NEED(s);
  *ms = s->e->last_iterate_ms;
  return DCFR_OK;
}

int dcfr_iteration_bytes(const dcfr_solver* s, double* bytes) {
  NEED(s);
  *bytes = s->e->iteration_bytes();
  return DCFR_OK;
}

int dcfr_last_solve_ms(const dcfr_solver* s, double* ms) {
  NEED(s);
  if (!ms) return fail(DCFR_ERR_INVALID_ARG, "NULL out");
  *ms = s->e->last_solve_ms;
  return DCFR_OK;
}

int dcfr_setup_profile_get(const dcfr_solver* s, dcfr_setup_profile* out) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "NULL out");
  *out = s->e->setup;
  return DCFR_OK;
}

int dcfr_terminal_kernel(const dcfr_solver* s, int32_t* kernel, int32_t* terminals_per_panel) {
  NEED(s);
  if (!kernel || !terminals_per_panel) return fail(DCFR_ERR_INVALID_ARG, "NULL out");
  s->e->terminal_kernel(*kernel, *terminals_per_panel);
  return DCFR_OK;
}

int dcfr_iterate_profiled(dcfr_solver* s, uint32_t iterations, dcfr_kernel_profile* out) {
  NEED(s);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  GUARD_BEGIN
  return done(s->e->iterate_profiled(iterations, *out));
  GUARD_END
}

// ------------------------------------------------------------ batched rivers
#define NEEDB(h)                                                      \
  if (!(h) || !(h)->b) return fail(DCFR_ERR_INVALID_ARG, "NULL batch")

int dcfr_batch_create(const dcfr_config* cfgs, int32_t count, dcfr_batch** out) {
  if (!cfgs || !out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *out = nullptr;
  GUARD_BEGIN
  std::unique_ptr<dcfr::Batch> b;
  dcfr::Status st = dcfr::Batch::create(cfgs, count, b);
  if (!st.ok()) return done(st);
  *out = new dcfr_batch{std::move(b)};
  g_error.clear();
  return DCFR_OK;
  GUARD_END
}

void dcfr_batch_destroy(dcfr_batch* b) { delete b; }

int dcfr_batch_iterate(dcfr_batch* b, uint32_t n) {
  NEEDB(b);
  GUARD_BEGIN
  return done(b->b->iterate(n));
  GUARD_END
}

int dcfr_batch_exploitability(dcfr_batch* b, double* out) {
  NEEDB(b);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  GUARD_BEGIN
  return done(b->b->exploitability(out));
  GUARD_END
}

int dcfr_batch_storage_len(const dcfr_batch* b, int32_t spot, uint64_t* len) {
  NEEDB(b);
  if (!len) return fail(DCFR_ERR_INVALID_ARG, "len is NULL");
  return done(b->b->storage_len(spot, *len));
}

int dcfr_batch_download_storage(dcfr_batch* b, int32_t spot, float* regrets, float* sums, uint64_t len) {
  NEEDB(b);
  uint64_t need = 0;
  dcfr::Status st = b->b->storage_len(spot, need);
  if (!st.ok()) return done(st);
  if (len < need) return fail(DCFR_ERR_INVALID_ARG, "storage buffers are too short");
  GUARD_BEGIN
  return done(b->b->download(spot, regrets, sums));
  GUARD_END
}

int dcfr_batch_autotune(dcfr_batch* b, uint32_t trial_iterations, dcfr_batch_tuning* out) {
  NEEDB(b);
  GUARD_BEGIN
  dcfr_batch_tuning best{};
  dcfr::Status st = b->b->autotune(trial_iterations, best);
  if (st.ok() && out) *out = best;
  return done(st);
  GUARD_END
}

int dcfr_batch_get_tuning(const dcfr_batch* b, dcfr_batch_tuning* out) {
  NEEDB(b);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  *out = b->b->tuning();
  return DCFR_OK;
}

int dcfr_batch_set_tuning(dcfr_batch* b, const dcfr_batch_tuning* t) {
  NEEDB(b);
  if (!t) return fail(DCFR_ERR_INVALID_ARG, "tuning is NULL");
  GUARD_BEGIN
  return done(b->b->set_tuning(*t));
  GUARD_END
}

int dcfr_batch_last_iterate_ms(const dcfr_batch* b, double* ms) {
  NEEDB(b);
  if (!ms) return fail(DCFR_ERR_INVALID_ARG, "ms is NULL");
  *ms = b->b->last_iterate_ms();
  return DCFR_OK;
}

int dcfr_batch_iterations(const dcfr_batch* b, uint32_t* out) {
  NEEDB(b);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  *out = b->b->iterations();
  return DCFR_OK;
}

int dcfr_batch_iteration_bytes(const dcfr_batch* b, double* bytes) {
  NEEDB(b);
  if (!bytes) return fail(DCFR_ERR_INVALID_ARG, "bytes is NULL");
  *bytes = b->b->iteration_bytes();
  return DCFR_OK;
}

int dcfr_batch_kernel_launches(const dcfr_batch* b, uint64_t* out) {
  NEEDB(b);
  if (!out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  *out = b->b->kernel_launches();
  return DCFR_OK;
}

}  // extern "C"
