// TEST INFRASTRUCTURE — C API of the CPU oracle for the Python tests and the
// CPU-baseline leg of bench.py (loaded with ctypes as oracle/liboracle.so).
// It takes the same dcfr_config layout as libdcfr (include/dcfr.h) so both
// sides are fed from one Python config object.
#include <cstring>
#include <string>

#include "../include/dcfr.h"
#include "solver.hpp"

using namespace oracle;

static thread_local std::string g_err;

static void fill_sizes(const dcfr_street_sizes& in, StreetSizes& out) {
  out.bet.clear();
  out.raise.clear();
  for (int i = 0; i < in.n_bet && i < DCFR_MAX_SIZES; i++) out.bet.push_back(BetSize{in.bet[i].kind, in.bet[i].value});
  for (int i = 0; i < in.n_raise && i < DCFR_MAX_SIZES; i++)
    out.raise.push_back(BetSize{in.raise[i].kind, in.raise[i].value});
}

static PostflopMenu to_menu(const dcfr_menu& m) {
  PostflopMenu out;
  fill_sizes(m.flop, out.flop);
  fill_sizes(m.turn, out.turn);
  fill_sizes(m.river, out.river);
  out.max_raises = m.max_raises;
  out.add_allin_threshold = m.add_allin_threshold;
  out.force_allin_threshold = m.force_allin_threshold;
  out.merge_threshold = m.merge_threshold;
  return out;
}

static BettingState to_state(const dcfr_betting_state& b) {
  BettingState s;
  s.street = (Street)b.street;
  s.pot = b.pot;
  s.commit[0] = b.commit[0];
  s.commit[1] = b.commit[1];
  s.stack[0] = b.stack[0];
  s.stack[1] = b.stack[1];
  s.current_bet = b.current_bet;
  s.last_raise_inc = b.last_raise_inc;
  s.num_raises = b.num_raises;
  s.to_act = b.to_act;
  s.needs[0] = b.needs[0] != 0;
  s.needs[1] = b.needs[1] != 0;
  return s;
}

static SolveConfig to_config(const dcfr_config* c) {
  SolveConfig cfg;
  for (int i = 0; i < c->board_len && i < 5; i++) cfg.board.push_back(c->board[i]);
  for (int p = 0; p < 2; p++) cfg.ranges[p].assign(c->ranges[p], c->ranges[p] + 1326);
  cfg.root = to_state(c->root);
  cfg.menu = to_menu(c->menu);
  cfg.has_future_menu = c->has_future_menu != 0;
  if (cfg.has_future_menu) cfg.future_menu = to_menu(c->future_menu);
  cfg.big_blind = c->big_blind;
  cfg.prune = c->prune;
  for (int p = 0; p < 2; p++)
    for (int i = 0; i < c->n_keep[p] && i < 1326; i++) cfg.keep[p].push_back(c->keep[p][i]);
  cfg.max_memory_bytes = c->max_memory_bytes;
  cfg.rake_rate = c->rake_rate;
  cfg.rake_cap = c->rake_cap;
  cfg.storage = c->storage;
  cfg.isomorphism = c->isomorphism != 0;
  cfg.dcfr.alpha = c->dcfr.alpha;
  cfg.dcfr.beta = c->dcfr.beta;
  cfg.dcfr.beta_clip = c->dcfr.beta_clip != 0;
  cfg.dcfr.gamma = c->dcfr.gamma;
  cfg.dcfr.restart_average = c->dcfr.restart_average != 0;
  cfg.dcfr.unweighted_average = c->dcfr.unweighted_average != 0;
  cfg.sampled = c->chance == DCFR_CHANCE_SAMPLED;
  cfg.sample_turn = (size_t)c->chance_turn;
  cfg.sample_river = (size_t)c->chance_river;
  cfg.sample_seed = c->chance_seed;
  return cfg;
}

static std::vector<Step> to_path(const dcfr_step* path, size_t n) {
  std::vector<Step> out;
  for (size_t i = 0; i < n; i++)
    out.push_back(Step{path[i].kind, Action{path[i].action_kind, path[i].amount}, (int)path[i].card});
  return out;
}

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

// The sampled chance mode's pieces, for the tests that pin them.
void oracle_chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
  chacha_block(key, counter, stream, rounds, out);
}
void oracle_rng_u64(uint64_t seed, uint64_t n, uint64_t* out) {
  ChaChaRng r(seed);
  for (uint64_t i = 0; i < n; i++) out[i] = r.next_u64();
}
int oracle_sample_cards(const int32_t* available, int32_t n, int32_t k, uint64_t seed, int32_t* out) {
  ChaChaRng r(seed);
  std::vector<int> a(available, available + n);
  std::vector<int> picks = sample_cards(a, (size_t)k, r);
  for (size_t i = 0; i < picks.size(); i++) out[i] = picks[i];
  return (int)picks.size();
}
void oracle_set_threads(int n) { set_num_threads(n); }
int oracle_get_threads(void) { return get_num_threads(); }

int oracle_estimate(const dcfr_config* c, dcfr_tree_stats* out) {
  TreeStats st;
  int err = 0;
  if (!Solver::estimate(to_config(c), st, err, g_err)) return err;
  out->player_nodes = st.player_nodes;
  out->chance_nodes = st.chance_nodes;
  out->terminal_nodes = st.terminal_nodes;
  out->storage_cells = st.storage_cells;
  out->compressed = st.compressed;
  out->memory_bytes = st.memory_bytes();
  return 0;
}

void* oracle_create(const dcfr_config* c, int* err) {
  int e = 0;
  auto s = Solver::create(to_config(c), e, g_err);
  *err = e;
  return s.release();
}

void oracle_destroy(void* h) { delete (Solver*)h; }

void oracle_set_batch_river(void* h, int on) { ((Solver*)h)->batch_river = on != 0; }

uint64_t oracle_storage_len(void* h) { return ((Solver*)h)->tree.storage_len; }
int oracle_is_compressed(void* h) { return ((Solver*)h)->store.compressed ? 1 : 0; }
uint64_t oracle_num_slots(void* h) { return ((Solver*)h)->tree.num_player_nodes; }
// Compressed storage (storage.rs:92-97): i16 regrets, u16 sums, per-slot scales.
int oracle_get_storage_compressed(void* h, int16_t* rq, uint16_t* sq, float* rscale, float* sscale) {
  const Solver* s = (const Solver*)h;
  if (!s->store.compressed) return 1;
  std::memcpy(rq, s->store.rq.data(), s->store.rq.size() * 2);
  std::memcpy(sq, s->store.sq.data(), s->store.sq.size() * 2);
  std::memcpy(rscale, s->store.rscale.data(), s->store.rscale.size() * 4);
  std::memcpy(sscale, s->store.sscale.data(), s->store.sscale.size() * 4);
  return 0;
}
int oracle_set_storage_compressed(void* h, const int16_t* rq, const uint16_t* sq, const float* rscale,
                                  const float* sscale) {
  Solver* s = (Solver*)h;
  if (!s->store.compressed) return 1;
  std::memcpy(s->store.rq.data(), rq, s->store.rq.size() * 2);
  std::memcpy(s->store.sq.data(), sq, s->store.sq.size() * 2);
  std::memcpy(s->store.rscale.data(), rscale, s->store.rscale.size() * 4);
  std::memcpy(s->store.sscale.data(), sscale, s->store.sscale.size() * 4);
  return 0;
}

void oracle_get_storage(void* h, float* regrets, float* sums) {
  Solver* s = (Solver*)h;
  std::memcpy(regrets, s->store.regrets.data(), s->store.regrets.size() * 4);
  std::memcpy(sums, s->store.strat.data(), s->store.strat.size() * 4);
}

void oracle_set_storage(void* h, const float* regrets, const float* sums) {
  Solver* s = (Solver*)h;
  std::memcpy(s->store.regrets.data(), regrets, s->store.regrets.size() * 4);
  std::memcpy(s->store.strat.data(), sums, s->store.strat.size() * 4);
}

void oracle_set_iterations(void* h, uint32_t t) { ((Solver*)h)->iterations = t; }
uint32_t oracle_iterations(void* h) { return ((Solver*)h)->iterations; }

int oracle_hands(void* h, int p, uint16_t* combos, float* weights) {
  Solver* s = (Solver*)h;
  int n = (int)s->hands.len(p);
  if (combos) std::memcpy(combos, s->hands.combos[p].data(), n * 2);
  if (weights) std::memcpy(weights, s->hands.weights[p].data(), n * 4);
  return n;
}

void oracle_stats(void* h, dcfr_tree_stats* out) {
  Solver* s = (Solver*)h;
  out->player_nodes = s->stats.player_nodes;
  out->chance_nodes = s->stats.chance_nodes;
  out->terminal_nodes = s->stats.terminal_nodes;
  out->storage_cells = s->stats.storage_cells;
  out->compressed = s->stats.compressed;
  out->memory_bytes = s->stats.memory_bytes();
}

int oracle_isomorphic_pairs(void* h) {
  Solver* s = (Solver*)h;
  int k = 0;
  for (int i = 0; i < 6; i++) k += s->iso.range_symmetric[i];
  return k;
}

uint64_t oracle_num_nodes(void* h) { return ((Solver*)h)->tree.nodes.size(); }

// Node table dump for the plan tests: per node kind, player, street,
// num_children, first_child, invest[2], offset, slot, rake, chance_factor,
// edge card, edge action kind/amount.
void oracle_nodes(void* h, int32_t* ints, uint64_t* offsets, float* floats, int64_t* amounts) {
  Solver* s = (Solver*)h;
  for (size_t i = 0; i < s->tree.nodes.size(); i++) {
    const Node& n = s->tree.nodes[i];
    int32_t* r = ints + i * 9;
    r[0] = n.kind;
    r[1] = n.player;
    r[2] = n.street;
    r[3] = n.num_children;
    r[4] = (int32_t)n.first_child;
    r[5] = n.invest[0];
    r[6] = n.invest[1];
    r[7] = n.edge_card;
    r[8] = n.edge_action.kind;
    offsets[i * 2] = n.offset;
    offsets[i * 2 + 1] = n.slot;
    floats[i * 2] = n.rake;
    floats[i * 2 + 1] = n.chance_factor;
    amounts[i] = n.edge_action.amount;
  }
}

void oracle_iterate(void* h, uint32_t n) { ((Solver*)h)->iterate(n); }

// n iterations of each of count independent solvers, spread over `threads`
// host threads (one solver per thread at a time, largest first as given):
// the CPU counterpart of the batched river solve.
void oracle_batch_iterate(void** hs, int count, uint32_t n, int threads) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
  for (int i = 0; i < count; i++) ((Solver*)hs[i])->iterate(n);
}

double oracle_exploitability(void* h) { return ((Solver*)h)->exploitability(); }

void oracle_root_values(void* h, double* out) { ((Solver*)h)->root_values(out); }

void oracle_traverse(void* h, int p, int mode, uint32_t t, float* out) { ((Solver*)h)->traverse_root(p, mode, t, out); }

typedef int (*oracle_cb)(const dcfr_progress*, void*);

int oracle_solve(void* h, const dcfr_solve_options* opts, oracle_cb cb, void* user, dcfr_progress* out) {
  Solver* s = (Solver*)h;
  std::function<bool(const Progress&)> f = [&](const Progress& p) {
    if (!cb) return true;
    dcfr_progress dp{p.iteration, p.max_iterations, p.exploitability, p.exploitability_pct, p.finished ? 1 : 0, 0};
    return cb(&dp, user) != 0;
  };
  Progress p = s->solve(opts->max_iterations, opts->target_exploitability_pct, opts->check_every, &f);
  out->iteration = p.iteration;
  out->max_iterations = p.max_iterations;
  out->exploitability = p.exploitability;
  out->exploitability_pct = p.exploitability_pct;
  out->finished = p.finished;
  return 0;
}

int oracle_query_sizes(void* h, const dcfr_step* path, size_t n, int32_t* na, int32_t* nh) {
  Solver* s = (Solver*)h;
  NodeInfo info;
  std::vector<Action> acts;
  if (!s->actions_at(to_path(path, n), acts, g_err)) return DCFR_ERR_BAD_PATH;
  if (!s->is_decision(to_path(path, n))) {
    g_err = "bad path: not a decision node";
    return DCFR_ERR_BAD_PATH;
  }
  // Player of the node: walk through query_sizes by a cheap query.
  *na = (int32_t)acts.size();
  // hands of the acting player
  std::string err;
  NodeInfo ni;
  if (!s->query(to_path(path, n), ni, err)) {
    g_err = err;
    return DCFR_ERR_BAD_PATH;
  }
  *nh = (int32_t)ni.combos.size();
  return 0;
}

int oracle_query(void* h, const dcfr_step* path, size_t n, dcfr_node_info* info, dcfr_action* actions,
                 uint16_t* combos, float* strategy, float* ev, float* reach) {
  Solver* s = (Solver*)h;
  NodeInfo ni;
  if (!s->query(to_path(path, n), ni, g_err)) return DCFR_ERR_BAD_PATH;
  info->player = ni.player;
  info->num_actions = (int32_t)ni.actions.size();
  info->num_hands = (int32_t)ni.combos.size();
  info->reach_fraction[0] = ni.reach_fraction[0];
  info->reach_fraction[1] = ni.reach_fraction[1];
  info->pot = ni.pot;
  info->invest[0] = ni.invest[0];
  info->invest[1] = ni.invest[1];
  for (size_t a = 0; a < ni.actions.size(); a++) actions[a] = dcfr_action{ni.actions[a].kind, 0, ni.actions[a].amount};
  std::memcpy(combos, ni.combos.data(), ni.combos.size() * 2);
  std::memcpy(strategy, ni.strategy.data(), ni.strategy.size() * 4);
  std::memcpy(ev, ni.ev.data(), ni.ev.size() * 4);
  std::memcpy(reach, ni.reach.data(), ni.reach.size() * 4);
  return 0;
}

int oracle_ranges_after(void* h, const dcfr_step* path, size_t n, float* out) {
  Solver* s = (Solver*)h;
  std::vector<float> r[2];
  if (!s->ranges_after(to_path(path, n), r, g_err)) return DCFR_ERR_BAD_PATH;
  std::memcpy(out, r[0].data(), 1326 * 4);
  std::memcpy(out + 1326, r[1].data(), 1326 * 4);
  return 0;
}

int oracle_actions_at(void* h, const dcfr_step* path, size_t n, dcfr_action* out, size_t cap, size_t* count) {
  Solver* s = (Solver*)h;
  std::vector<Action> acts;
  if (!s->actions_at(to_path(path, n), acts, g_err)) return DCFR_ERR_BAD_PATH;
  *count = acts.size();
  for (size_t i = 0; i < acts.size() && i < cap; i++) out[i] = dcfr_action{acts[i].kind, 0, acts[i].amount};
  return 0;
}

int oracle_is_decision(void* h, const dcfr_step* path, size_t n) {
  return ((Solver*)h)->is_decision(to_path(path, n)) ? 1 : 0;
}

// ------------------------------------------------------------ primitives
uint32_t oracle_evaluate(const int32_t* cards, int n) {
  int c[7];
  for (int i = 0; i < n && i < 7; i++) c[i] = cards[i];
  return evaluate_cards(c, n);
}

// All 2,598,960 five-card hands, counted per category
// (crates/holdem/src/eval.rs:246-265).
void oracle_five_card_counts(uint32_t* out9) {
  for (int i = 0; i < 9; i++) out9[i] = 0;
  for (int a = 0; a < 52; a++)
    for (int b = a + 1; b < 52; b++)
      for (int c = b + 1; c < 52; c++)
        for (int d = c + 1; d < 52; d++) {
          uint64_t m4 = eval_card_bit(a) | eval_card_bit(b) | eval_card_bit(c) | eval_card_bit(d);
          for (int e = d + 1; e < 52; e++) out9[evaluate_mask(m4 | eval_card_bit(e)) >> 26]++;
        }
}

int oracle_combo_index(int a, int b) { return combo_index(a, b); }

void oracle_combos(uint8_t* hi_lo) {
  for (int i = 0; i < 1326; i++) {
    hi_lo[2 * i] = combos_table()[i].hi;
    hi_lo[2 * i + 1] = combos_table()[i].lo;
  }
}

void oracle_combo_class(uint8_t* out) { std::memcpy(out, combo_class_table(), 1326); }

int oracle_class_combos(int grid_index, int32_t* out) {
  auto v = HandClass::from_grid_index(grid_index).combos();
  for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
  return (int)v.size();
}

int oracle_parse_range(const char* s, float* out1326) {
  std::vector<float> w;
  if (!parse_range(s, w, &g_err)) return DCFR_ERR_INVALID_ARG;
  std::memcpy(out1326, w.data(), 1326 * 4);
  return 0;
}

int oracle_parse_cards(const char* s, int32_t* out, int cap) {
  std::vector<int> c;
  if (!parse_cards(s, c)) return -1;
  for (size_t i = 0; i < c.size() && (int)i < cap; i++) out[i] = c[i];
  return (int)c.size();
}

int oracle_menu_actions(const dcfr_menu* menu, int street, int64_t pot, int64_t to_call, int64_t current_bet,
                        int64_t max_to, int64_t min_raise_to, uint32_t num_raises, int64_t big_blind, dcfr_action* out,
                        int cap) {
  Situation sit{(Street)street, pot, to_call, current_bet, max_to, min_raise_to, num_raises, big_blind};
  auto acts = postflop_actions(sit, to_menu(*menu));
  for (size_t i = 0; i < acts.size() && (int)i < cap; i++) out[i] = dcfr_action{acts[i].kind, 0, acts[i].amount};
  return (int)acts.size();
}

void oracle_default_menu(dcfr_menu* out) {
  PostflopMenu m = PostflopMenu::defaults();
  std::memset(out, 0, sizeof *out);
  auto put = [](const StreetSizes& s, dcfr_street_sizes& d) {
    d.n_bet = (int)s.bet.size();
    d.n_raise = (int)s.raise.size();
    for (size_t i = 0; i < s.bet.size(); i++) d.bet[i] = dcfr_bet_size{s.bet[i].kind, 0, s.bet[i].value};
    for (size_t i = 0; i < s.raise.size(); i++) d.raise[i] = dcfr_bet_size{s.raise[i].kind, 0, s.raise[i].value};
  };
  put(m.flop, out->flop);
  put(m.turn, out->turn);
  put(m.river, out->river);
  out->max_raises = m.max_raises;
  out->add_allin_threshold = m.add_allin_threshold;
  out->force_allin_threshold = m.force_allin_threshold;
  out->merge_threshold = m.merge_threshold;
}

int oracle_parse_bet_size(const char* s, int32_t* kind, double* value) {
  BetSize b;
  if (!parse_bet_size(s, b)) return -1;
  *kind = b.kind;
  *value = b.value;
  return 0;
}

uint32_t oracle_next_check_gap(int has_prev, uint32_t t0, double e0, uint32_t t, double e, double target,
                               uint32_t max_gap) {
  return next_check_gap(has_prev != 0, t0, e0, t, e, target, max_gap);
}

void oracle_discount(uint32_t t, const dcfr_params* p, float* out3) {
  DcfrParams d;
  d.alpha = p->alpha;
  d.beta = p->beta;
  d.beta_clip = p->beta_clip != 0;
  d.gamma = p->gamma;
  d.restart_average = p->restart_average != 0;
  d.unweighted_average = p->unweighted_average != 0;
  Discount x = Discount::make(t, d);
  out3[0] = x.pos;
  out3[1] = x.neg;
  out3[2] = x.strat;
}

int oracle_board_symmetric_pairs(const int32_t* board, int n, int32_t* out_pairs) {
  std::vector<int> b(board, board + n);
  auto v = board_symmetric_pairs(b);
  for (size_t i = 0; i < v.size(); i++) {
    out_pairs[2 * i] = v[i].first;
    out_pairs[2 * i + 1] = v[i].second;
  }
  return (int)v.size();
}

int oracle_iso_orbit(const int32_t* board, int n, int combo, int32_t* out) {
  std::vector<int> b(board, board + n);
  auto v = iso_orbit(b, combo);
  for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
  return (int)v.size();
}

// ------------------------------------------------------------ evaluators
struct HS {
  HandSet hs;
  std::vector<int> board;
  StrengthTable table;
};

void* oracle_handset_create(const float* r0, const float* r1, const int32_t* board, int nb) {
  HS* h = new HS();
  std::vector<float> r[2] = {std::vector<float>(r0, r0 + 1326), std::vector<float>(r1, r1 + 1326)};
  uint64_t set = 0;
  for (int i = 0; i < nb; i++) {
    set |= 1ull << board[i];
    h->board.push_back(board[i]);
  }
  std::vector<int> keep[2];
  h->hs.build(r, set, 0.0f, keep);
  if (nb == 5) h->table.build(h->hs, h->board);
  return h;
}

void oracle_handset_destroy(void* h) { delete (HS*)h; }
int oracle_handset_len(void* h, int p) { return (int)((HS*)h)->hs.len(p); }
double oracle_handset_num_combinations(void* h) { return ((HS*)h)->hs.num_combinations; }
void oracle_handset_cards(void* h, int p, uint8_t* out) {
  HS* x = (HS*)h;
  for (size_t i = 0; i < x->hs.len(p); i++) {
    out[2 * i] = x->hs.cards[p][i].first;
    out[2 * i + 1] = x->hs.cards[p][i].second;
  }
}

void oracle_compatible_reach(void* h, int p, const float* r, double* out) {
  auto v = ((HS*)h)->hs.compatible_reach(p, r);
  std::memcpy(out, v.data(), v.size() * 8);
}

void oracle_eval_fold(void* h, int p, const float* r, double payoff, float* out) {
  eval_fold(((HS*)h)->hs, p, r, payoff, out);
}

void oracle_eval_showdown(void* h, int p, const float* r, double w, double l, double t, float* out) {
  HS* x = (HS*)h;
  eval_showdown(x->hs, x->table, p, r, w, l, t, out);
}

void oracle_fold_batch(void* h, int p, int k, const float* const* reaches, const double* payoffs, float* const* outs) {
  std::vector<const float*> rs(reaches, reaches + k);
  std::vector<double> ps(payoffs, payoffs + k);
  std::vector<float*> os(outs, outs + k);
  fold_batch(((HS*)h)->hs, p, rs, ps, os);
}

void oracle_showdown_batch(void* h, int p, int k, const float* const* reaches, const double* win, const double* lose,
                           const double* tie, float* const* outs, const double* fold_pay, float* const* fold_outs) {
  HS* x = (HS*)h;
  std::vector<const float*> rs(reaches, reaches + k);
  std::vector<double> w(win, win + k), l(lose, lose + k), t(tie, tie + k);
  std::vector<float*> os(outs, outs + k);
  std::vector<std::pair<double, float*>> folds;
  std::vector<bool> has;
  for (int i = 0; i < k; i++) {
    folds.push_back({fold_pay ? fold_pay[i] : 0.0, fold_outs ? fold_outs[i] : nullptr});
    has.push_back(fold_outs && fold_outs[i] != nullptr);
  }
  showdown_batch(x->hs, x->table, p, rs, w, l, t, os, folds, has);
}

}  // extern "C"
