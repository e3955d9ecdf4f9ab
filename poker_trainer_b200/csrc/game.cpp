// Host-side game model of libdcfr (see game.hpp).
#include "game.hpp"
#include "chance_sample.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace dcfr {

static inline int rank_of(int c) { return c >> 2; }
static inline int suit_of(int c) { return c & 3; }
static inline int combo_id(int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  return hi * (hi - 1) / 2 + lo;
}

std::vector<Act> Game::actions(uint32_t id) const {
  std::vector<Act> out;
  const GNode& nd = nodes[id];
  for (uint32_t c = nd.first; c < nd.first + nd.nchild; c++) out.push_back(nodes[c].act);
  return out;
}

uint64_t reference_memory_bytes(const Stats& s, bool compressed) {
  // Node is 56 bytes in the reference (tree.rs:154-171).
  return s.cells * (compressed ? 4 : 8) + (s.player + s.chance + s.terminal) * 56ull;
}

// ------------------------------------------------------------------ menu
static const dcfr_street_sizes& sizes_for(const dcfr_menu& m, int street) {
  return street == DCFR_TURN ? m.turn : street == DCFR_RIVER ? m.river : m.flop;
}

struct Amount {
  int64_t to;
  uint32_t tag;
};

// Clamp to [min raise, all-in], force near-all-in sizes to all-in, drop
// non-raises, sort by (amount, tag), keep one per amount, merge close sizes
// (finalize_tagged, menu.rs:355-392).
static void finalize(int64_t min_raise_to, int64_t max_to, int64_t pot_after_call, int64_t current_bet,
                     double force_allin, double merge, std::vector<Amount>& v) {
  int64_t lo = std::min(min_raise_to, max_to);
  std::vector<Amount> w;
  for (const Amount& x : v) {
    int64_t a = x.to < lo ? lo : (x.to > max_to ? max_to : x.to);
    int64_t new_pot = pot_after_call + 2 * (a - current_bet);
    int64_t thr = (int64_t)std::round((double)new_pot * force_allin);
    if (max_to - a <= thr) a = max_to;
    if (a > current_bet) w.push_back(Amount{a, x.tag});
  }
  std::sort(w.begin(), w.end(), [](const Amount& a, const Amount& b) {
    return a.to != b.to ? a.to < b.to : a.tag < b.tag;
  });
  v.clear();
  for (const Amount& x : w)
    if (v.empty() || v.back().to != x.to) v.push_back(x);
  if (merge > 0.0 && v.size() > 1) {
    auto ratio = [&](int64_t a) { return (double)(a - current_bet) / (double)pot_after_call; };
    std::vector<Amount> kept;
    for (size_t i = v.size(); i-- > 0;) {
      if (!kept.empty() && (1.0 + ratio(kept.back().to)) / (1.0 + ratio(v[i].to)) < 1.0 + merge) continue;
      kept.push_back(v[i]);
    }
    std::reverse(kept.begin(), kept.end());
    v.swap(kept);
  }
}

std::vector<Act> state_actions(const Betting& st, const dcfr_menu& menu, int64_t big_blind) {
  // Situation (tree.rs:63-77).
  int p = st.to_act, o = p ^ 1;
  int64_t to_call = std::min(std::max(st.current_bet - st.commit[p], (int64_t)0), st.stack[p]);
  int64_t max_to = std::min(st.commit[p] + st.stack[p], st.commit[o] + st.stack[o]);
  int64_t min_raise_to = st.current_bet + std::max(st.last_raise_inc, big_blind);
  std::vector<Act> out;
  if (to_call > 0) {
    out.push_back(Act{DCFR_FOLD, 0});
    out.push_back(Act{DCFR_CALL, 0});
  } else {
    out.push_back(Act{DCFR_CHECK, 0});
  }
  if (!(max_to > st.current_bet) || st.num_raises >= menu.max_raises) return out;
  const dcfr_street_sizes& sz = sizes_for(menu, st.street);
  const dcfr_bet_size* list = st.current_bet == 0 ? sz.bet : sz.raise;
  int nlist = st.current_bet == 0 ? sz.n_bet : sz.n_raise;
  double pac = (double)(st.pot + to_call);
  std::vector<Amount> amounts;
  for (int i = 0; i < nlist; i++) {
    int64_t to;
    if (list[i].kind == DCFR_SIZE_POT) {
      to = st.current_bet + (int64_t)std::round(list[i].value * pac);
    } else if (list[i].kind == DCFR_SIZE_MULT) {
      if (st.current_bet == 0) continue;
      to = (int64_t)std::round(list[i].value * (double)st.current_bet);
    } else {
      to = max_to;
    }
    amounts.push_back(Amount{to, (uint32_t)i});
  }
  if (menu.add_allin_threshold > 0.0 && (double)(max_to - st.current_bet) <= menu.add_allin_threshold * pac)
    amounts.push_back(Amount{max_to, (uint32_t)nlist});
  finalize(min_raise_to, max_to, st.pot + to_call, st.current_bet, menu.force_allin_threshold, menu.merge_threshold,
           amounts);
  for (const Amount& a : amounts) out.push_back(Act{DCFR_RAISE, a.to});
  return out;
}

// BettingState::apply (tree.rs:93-125): 0 = continue, 1 = fold, 2 = street over.
static int apply(const Betting& st, const Act& a, Betting& s, int64_t& put) {
  int p = st.to_act, o = p ^ 1;
  s = st;
  put = 0;
  if (a.kind == DCFR_FOLD) return 1;
  if (a.kind == DCFR_CALL) {
    put = std::min(std::max(s.current_bet - s.commit[p], (int64_t)0), s.stack[p]);
  } else if (a.kind == DCFR_RAISE) {
    put = a.amount - s.commit[p];
    int64_t inc = a.amount - s.current_bet;
    if (inc >= s.last_raise_inc) s.last_raise_inc = inc;
    s.current_bet = a.amount;
    s.num_raises += 1;
    s.needs[o] = s.stack[o] > 0;
  }
  s.commit[p] += put;
  s.stack[p] -= put;
  s.pot += put;
  s.needs[p] = false;
  if (s.needs[o]) {
    s.to_act = o;
    return 0;
  }
  return 2;
}

static Betting street_start(int street, int64_t pot, int64_t s0, int64_t s1, int64_t bb) {
  Betting b;
  b.street = street;
  b.pot = pot;
  b.commit[0] = b.commit[1] = 0;
  b.stack[0] = s0;
  b.stack[1] = s1;
  b.current_bet = 0;
  b.last_raise_inc = bb;
  b.num_raises = 0;
  b.to_act = 0;
  b.needs[0] = s0 > 0;
  b.needs[1] = s1 > 0;
  return b;
}

// ------------------------------------------------------------------ iso
static const uint8_t PAIRS[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

static int pair_of(int a, int b) {
  if (a > b) std::swap(a, b);
  for (int i = 0; i < 6; i++)
    if (PAIRS[i][0] == a && PAIRS[i][1] == b) return i;
  return -1;
}

static int swapped(int card, int a, int b) {
  int s = suit_of(card);
  return rank_of(card) * 4 + (s == a ? b : s == b ? a : s);
}

// ------------------------------------------------------------------ tree
struct Ctx {
  Game* g;
  const dcfr_menu* menu;
  const dcfr_menu* future;
  int root_street;
  int64_t bb;
  std::unordered_map<uint64_t, uint32_t> board_index;
  StdRng* rng = nullptr;  // the sampled chance mode's generator

  const dcfr_menu& menu_for(int street) const { return street == root_street ? *menu : *future; }
  // The action list of a betting state (state_actions), memoised: a tree
  // repeats the same few hundred states once per dealt card, and the list
  // depends on nothing else (the menu and big blind are fixed per build).
  struct StateKey {
    int64_t v[8];
    bool operator==(const StateKey& o) const { return std::memcmp(v, o.v, sizeof v) == 0; }
  };
  struct StateHash {
    size_t operator()(const StateKey& k) const {
      uint64_t h = 1469598103934665603ull;
      for (int64_t x : k.v) h = (h ^ (uint64_t)x) * 1099511628211ull;
      return (size_t)h;
    }
  };
  mutable std::unordered_map<StateKey, std::vector<Act>, StateHash> act_cache;
  const std::vector<Act>& acts(const Betting& st) const {
    const StateKey k{{(int64_t)st.street | (int64_t)st.to_act << 8 | (int64_t)st.num_raises << 16, st.pot,
                      st.commit[0], st.commit[1], st.stack[0], st.stack[1], st.current_bet, st.last_raise_inc}};
    auto it = act_cache.find(k);
    if (it == act_cache.end()) it = act_cache.emplace(k, state_actions(st, menu_for(st.street), bb)).first;
    return it->second;
  }
  float rake(int64_t pot) const {
    return (float)std::min((double)pot * g->cfg.rake_rate, g->cfg.rake_cap);
  }
  // Canonical cards and isomorphic references dealt at a chance node
  // (tree.rs:315-334, iso.rs:120-141). In the sampled chance mode a chance
  // node that is not an all-in runout deals a stratified sample of the
  // street's size instead, with no isomorphic references.
  void deal(const std::vector<int>& dealt, bool all_in, int next, std::vector<int>& canon,
            std::vector<int>& iso_card, std::vector<int>& iso_canon, std::vector<int>& iso_pair,
            int& n_avail) const {
    uint64_t used = 0;
    uint16_t m[4] = {0, 0, 0, 0};
    for (int c : g->board) {
      used |= 1ull << c;
      m[suit_of(c)] |= (uint16_t)(1u << rank_of(c));
    }
    for (int c : dealt) {
      used |= 1ull << c;
      m[suit_of(c)] |= (uint16_t)(1u << rank_of(c));
    }
    canon.clear();
    iso_card.clear();
    iso_canon.clear();
    iso_pair.clear();
    n_avail = 52 - __builtin_popcountll(used);
    if (g->cfg.chance == DCFR_CHANCE_SAMPLED && !all_in) {
      const size_t k = (size_t)(next == DCFR_TURN ? g->cfg.chance_turn : g->cfg.chance_river);
      if (k < (size_t)n_avail) {
        std::vector<int> available;
        for (int c = 0; c < 52; c++)
          if (!(used >> c & 1)) available.push_back(c);
        canon = sample_cards(available, k, *rng);
        return;
      }
    }
    n_avail = 0;
    bool any = false;
    for (int i = 0; i < 6; i++) any |= g->sym[i];
    for (int c = 0; c < 52; c++) {
      if (used >> c & 1) continue;
      n_avail++;
      int s = suit_of(c), found = -1;
      if (g->iso_enabled && any)
        for (int s0 = 0; s0 < s; s0++)
          if (g->sym[pair_of(s0, s)] && m[s0] == m[s]) {
            found = s0;
            break;
          }
      if (found >= 0) {
        iso_card.push_back(c);
        iso_canon.push_back(rank_of(c) * 4 + found);
        iso_pair.push_back(pair_of(found, s));
      } else {
        canon.push_back(c);
      }
    }
  }
};

static void count_street_over(Ctx& cx, const Betting& st, std::vector<int>& dealt, Stats& s);

static void count_player(Ctx& cx, const Betting& st, std::vector<int>& dealt, Stats& s) {
  s.player++;
  const std::vector<Act>& acts = cx.acts(st);
  s.cells += (uint64_t)acts.size() * (uint64_t)cx.g->n[st.to_act];
  for (const Act& a : acts) {
    Betting s2;
    int64_t put;
    int tr = apply(st, a, s2, put);
    if (tr == 0)
      count_player(cx, s2, dealt, s);
    else if (tr == 1)
      s.terminal++;
    else
      count_street_over(cx, s2, dealt, s);
  }
}

// count_after_street (tree.rs:364-401): without isomorphism every runout's
// subtree has the same size, so one stands for all.
static void count_street_over(Ctx& cx, const Betting& st, std::vector<int>& dealt, Stats& s) {
  if (st.street == DCFR_RIVER || (cx.g->leaf_street >= 0 && st.street + 1 >= cx.g->leaf_street)) {
    s.terminal++;
    return;
  }
  s.chance++;
  bool all_in = st.stack[0] == 0 || st.stack[1] == 0;
  std::vector<int> canon, ic, icn, ip;
  int n_avail;
  cx.deal(dealt, all_in, st.street + 1, canon, ic, icn, ip, n_avail);
  bool uniform = ic.empty() && !cx.g->iso_enabled;
  size_t reps = uniform ? 1 : canon.size();
  Stats sub;
  for (size_t i = 0; i < reps; i++) {
    dealt.push_back(canon[i]);
    if (all_in) {
      Betting s2 = st;
      s2.street = st.street + 1;
      count_street_over(cx, s2, dealt, sub);
    } else {
      count_player(cx, street_start(st.street + 1, st.pot, st.stack[0], st.stack[1], cx.bb), dealt, sub);
    }
    dealt.pop_back();
  }
  uint64_t k = uniform ? canon.size() : 1;
  s.player += sub.player * k;
  s.chance += sub.chance * k;
  s.terminal += sub.terminal * k;
  s.cells += sub.cells * k;
}

static void fill_street_over(Ctx& cx, uint32_t id, const Betting& st, int32_t i0, int32_t i1, std::vector<int>& dealt);

// Builder::fill_player (tree.rs:451-499).
static void fill_player(Ctx& cx, uint32_t id, const Betting& st, int32_t i0, int32_t i1, std::vector<int>& dealt) {
  Game& g = *cx.g;
  const std::vector<Act>& acts = cx.acts(st);
  uint32_t first = (uint32_t)g.nodes.size();
  g.nodes.resize(g.nodes.size() + acts.size());
  GNode& nd = g.nodes[id];
  nd.kind = N_PLAYER;
  nd.player = (uint8_t)st.to_act;
  nd.street = (uint8_t)st.street;
  nd.nchild = (uint16_t)acts.size();
  nd.first = first;
  nd.invest[0] = i0;
  nd.invest[1] = i1;
  nd.ref_offset = g.storage_len;
  nd.index = g.player_nodes;
  g.storage_len += (uint64_t)acts.size() * (uint64_t)g.n[st.to_act];
  g.player_nodes++;
  for (size_t i = 0; i < acts.size(); i++) {
    uint32_t child = first + (uint32_t)i;
    Betting s2;
    int64_t put;
    int tr = apply(st, acts[i], s2, put);
    int32_t inv[2] = {i0, i1};
    inv[st.to_act] += (int32_t)put;
    g.nodes[child].act = acts[i];
    g.nodes[child].parent = id;
    if (tr == 0) {
      fill_player(cx, child, s2, inv[0], inv[1], dealt);
    } else if (tr == 1) {
      int f = st.to_act, o = f ^ 1;
      int64_t uncalled = std::max(st.commit[o] - st.commit[f], (int64_t)0);
      GNode& t = g.nodes[child];
      t.kind = N_FOLD;
      t.player = (uint8_t)f;
      t.street = (uint8_t)st.street;
      t.invest[0] = inv[0];
      t.invest[1] = inv[1];
      t.rake = cx.rake(st.pot - uncalled);
    } else {
      fill_street_over(cx, child, s2, inv[0], inv[1], dealt);
    }
  }
}

// Builder::fill_after_street (tree.rs:501-560) and table_for (562-573).
static void fill_street_over(Ctx& cx, uint32_t id, const Betting& st, int32_t i0, int32_t i1, std::vector<int>& dealt) {
  Game& g = *cx.g;
  if (g.leaf_street >= 0 && st.street + 1 >= g.leaf_street && st.street != DCFR_RIVER) {
    GNode& nd = g.nodes[id];
    nd.kind = N_LEAF;
    nd.street = (uint8_t)st.street;
    nd.invest[0] = i0;
    nd.invest[1] = i1;
    nd.index = (uint32_t)g.leaves.size();
    g.leaves.push_back(Game::Leaf{id, st.pot, std::min(st.stack[0], st.stack[1])});
    return;
  }
  if (st.street == DCFR_RIVER) {
    uint64_t key = 0;
    for (int c : dealt) key |= 1ull << c;
    uint32_t table;
    auto it = cx.board_index.find(key);
    if (it != cx.board_index.end()) {
      table = it->second;
    } else {
      table = (uint32_t)g.boards.size();
      std::vector<int> b = g.board;
      b.insert(b.end(), dealt.begin(), dealt.end());
      g.boards.push_back(b);
      cx.board_index[key] = table;
    }
    GNode& nd = g.nodes[id];
    nd.kind = N_SHOWDOWN;
    nd.street = DCFR_RIVER;
    nd.invest[0] = i0;
    nd.invest[1] = i1;
    nd.index = table;
    nd.rake = cx.rake(st.pot);
    return;
  }
  bool all_in = st.stack[0] == 0 || st.stack[1] == 0;
  std::vector<int> canon, ic, icn, ip;
  int n_avail;
  cx.deal(dealt, all_in, st.street + 1, canon, ic, icn, ip, n_avail);
  size_t board_len = g.board.size() + dealt.size();
  float compatible = (float)(52 - board_len - 4);
  size_t total_cards = canon.size() + ic.size();
  uint32_t first = (uint32_t)g.nodes.size();
  g.nodes.resize(g.nodes.size() + canon.size());
  ChanceIso info;
  for (size_t r = 0; r < ic.size(); r++) {
    size_t k = std::find(canon.begin(), canon.end(), icn[r]) - canon.begin();
    info.ci.push_back((uint16_t)k);
    info.pair.push_back((uint8_t)ip[r]);
    info.cards.push_back((uint8_t)ic[r]);
  }
  uint32_t ord = (uint32_t)g.chance.size();
  g.chance.push_back(info);
  GNode& nd = g.nodes[id];
  nd.kind = N_CHANCE;
  nd.street = (uint8_t)st.street;
  nd.nchild = (uint16_t)canon.size();
  nd.first = first;
  nd.invest[0] = i0;
  nd.invest[1] = i1;
  nd.index = ord;
  // 1 / (cards * compatible / available), all f32 (tree.rs:542).
  float denom = (float)total_cards * compatible / (float)n_avail;
  nd.factor = 1.0f / denom;
  for (size_t i = 0; i < canon.size(); i++) {
    uint32_t child = first + (uint32_t)i;
    g.nodes[child].card = canon[i];
    g.nodes[child].parent = id;
    dealt.push_back(canon[i]);
    if (all_in) {
      Betting s2 = st;
      s2.street = st.street + 1;
      fill_street_over(cx, child, s2, i0, i1, dealt);
    } else {
      fill_player(cx, child, street_start(st.street + 1, st.pot, st.stack[0], st.stack[1], cx.bb), i0, i1, dealt);
    }
    dealt.pop_back();
  }
}

// ------------------------------------------------------------------ hands
static void build_hands(Game& g, uint64_t board_set) {
  const dcfr_config& c = g.cfg;
  for (int p = 0; p < 2; p++) {
    float max_w = 0.0f;
    for (int i = 0; i < DCFR_NUM_COMBOS; i++) max_w = std::max(max_w, c.ranges[p][i]);
    float cutoff = max_w * c.prune;
    g.combos[p].clear();
    g.c1[p].clear();
    g.c2[p].clear();
    g.weights[p].clear();
    int idx = 0;
    for (int id = 0; id < DCFR_NUM_COMBOS; id++) {
      // combo id -> (hi, lo) with hi*(hi-1)/2 + lo = id
      int hi = (int)((1.0 + std::sqrt(1.0 + 8.0 * id)) / 2.0);
      while (hi * (hi - 1) / 2 > id) hi--;
      while ((hi + 1) * hi / 2 <= id) hi++;
      int lo = id - hi * (hi - 1) / 2;
      if ((board_set >> hi & 1) || (board_set >> lo & 1)) continue;
      float w = c.ranges[p][id];
      bool forced = false;
      for (int k = 0; k < c.n_keep[p] && k < DCFR_NUM_COMBOS; k++)
        if (c.keep[p][k] == id) forced = true;
      if ((w > 0.0f && w >= cutoff) || (forced && w > 0.0f)) {
        g.combos[p].push_back((uint16_t)id);
        g.c1[p].push_back((uint8_t)hi);
        g.c2[p].push_back((uint8_t)lo);
        g.weights[p].push_back(w);
        idx++;
      }
    }
    g.n[p] = idx;
  }
  for (int p = 0; p < 2; p++) {
    g.lookup[p].assign(DCFR_NUM_COMBOS, NO);
    for (int i = 0; i < g.n[p]; i++) g.lookup[p][g.combos[p][i]] = (uint32_t)i;
    g.blocked[p].assign(52, {});
    for (int i = 0; i < g.n[p]; i++) {
      g.blocked[p][g.c1[p][i]].push_back((uint32_t)i);
      g.blocked[p][g.c2[p][i]].push_back((uint32_t)i);
    }
  }
  for (int p = 0; p < 2; p++) {
    g.same[p].resize(g.n[p]);
    for (int i = 0; i < g.n[p]; i++) g.same[p][i] = g.lookup[p ^ 1][g.combos[p][i]];
  }
  // Total weight of compatible pairs, f64 in hand order
  // (hands.rs:95-125).
  double total = 0.0, minus[52] = {0};
  for (int k = 0; k < g.n[1]; k++) {
    float w = g.weights[1][k];
    if (w != 0.0f) {
      total += (double)w;
      minus[g.c1[1][k]] += (double)w;
      minus[g.c2[1][k]] += (double)w;
    }
  }
  double s = -0.0;
  for (int i = 0; i < g.n[0]; i++) {
    double sw = g.same[0][i] == NO ? 0.0 : (double)g.weights[1][g.same[0][i]];
    double v = total - minus[g.c1[0][i]] - minus[g.c2[0][i]] + sw;
    s += (v > 0.0 ? v : 0.0) * (double)g.weights[0][i];
  }
  g.num_combinations = s;
}

static void build_iso(Game& g) {
  g.iso_enabled = g.cfg.isomorphism != 0;
  for (int pi = 0; pi < 6; pi++) {
    g.sym[pi] = false;
    g.perm[0][pi].clear();
    g.perm[1][pi].clear();
  }
  if (!g.iso_enabled) return;
  for (int pi = 0; pi < 6; pi++) {
    int a = PAIRS[pi][0], b = PAIRS[pi][1];
    std::vector<uint16_t> pp[2];
    bool ok = true;
    for (int p = 0; p < 2 && ok; p++) {
      float max_w = 0.0f;
      for (float x : g.weights[p]) max_w = std::max(max_w, x);
      max_w = std::max(max_w, 1e-30f);
      for (int h = 0; h < g.n[p] && ok; h++) {
        uint32_t j = g.lookup[p][combo_id(swapped(g.c1[p][h], a, b), swapped(g.c2[p][h], a, b))];
        if (j == NO || std::fabs(g.weights[p][h] - g.weights[p][j]) > 1e-4f * max_w) {
          ok = false;
          break;
        }
        pp[p].push_back((uint16_t)j);
      }
    }
    if (!ok) continue;
    g.sym[pi] = true;
    g.perm[0][pi] = pp[0];
    g.perm[1][pi] = pp[1];
  }
}

std::vector<uint32_t> players_in_storage_order(const Game& g) {
  std::vector<uint32_t> players((size_t)g.player_nodes);
  for (uint32_t v = 0; v < (uint32_t)g.nodes.size(); v++)
    if (g.nodes[v].kind == N_PLAYER) players[g.nodes[v].index] = v;
  return players;
}

void normalize_rows(float* s, int na, int n) {
  for (int h = 0; h < n; h++) {
    float d = s[h];
    for (int a = 1; a < na; a++) d += s[a * n + h];
    float i = 1.0f / d;
    float inv = (d > 0.0f && std::isfinite(i)) ? i : 0.0f;
    if (inv == 0.0f) {
      float u = 1.0f / (float)na;
      for (int a = 0; a < na; a++) s[a * n + h] = u;
    } else {
      for (int a = 0; a < na; a++) s[a * n + h] *= inv;
    }
  }
}

int build_game(const dcfr_config& cfg, Game& g, std::string& msg, bool build_tree, int leaf_street) {
  g.cfg = cfg;
  g.leaf_street = leaf_street;
  g.leaves.clear();
  int nb = cfg.board_len;
  if (nb < 3 || nb > 5) {
    msg = "invalid board: " + std::to_string(nb) + " cards";
    return DCFR_ERR_INVALID_BOARD;
  }
  uint64_t set = 0;
  g.board.clear();
  for (int i = 0; i < nb; i++) {
    if (cfg.board[i] >= 52) {
      msg = "invalid board: card id out of range";
      return DCFR_ERR_INVALID_BOARD;
    }
    set |= 1ull << cfg.board[i];
    g.board.push_back(cfg.board[i]);
  }
  if (__builtin_popcountll(set) != nb) {
    msg = "invalid board: duplicate cards";
    return DCFR_ERR_INVALID_BOARD;
  }
  int street = nb == 3 ? DCFR_FLOP : nb == 4 ? DCFR_TURN : DCFR_RIVER;
  if (street != cfg.root.street) {
    msg = "invalid board: board doesn't match the root street";
    return DCFR_ERR_INVALID_BOARD;
  }
  if (cfg.root.to_act < 0 || cfg.root.to_act > 1) {
    msg = "root.to_act must be 0 or 1";
    return DCFR_ERR_INVALID_ARG;
  }
  if (cfg.chance != DCFR_CHANCE_EXACT && cfg.chance != DCFR_CHANCE_SAMPLED) {
    msg = "chance must be DCFR_CHANCE_EXACT or DCFR_CHANCE_SAMPLED";
    return DCFR_ERR_INVALID_ARG;
  }
  if (cfg.chance == DCFR_CHANCE_SAMPLED) {
    if (cfg.chance_turn < 1 || cfg.chance_river < 1) {
      msg = "a sampled chance mode deals at least one card per street";
      return DCFR_ERR_INVALID_ARG;
    }
    if (leaf_street >= 0) {
      msg = "the depth-limited solver values every dealt card; the sampled chance mode is not built for it";
      return DCFR_ERR_UNSUPPORTED;
    }
  }
  for (const dcfr_menu* m : {&cfg.menu, &cfg.future_menu}) {
    for (const dcfr_street_sizes* s : {&m->flop, &m->turn, &m->river})
      if (s->n_bet < 0 || s->n_bet > DCFR_MAX_SIZES || s->n_raise < 0 || s->n_raise > DCFR_MAX_SIZES) {
        msg = "a street has more than 8 sizes";
        return DCFR_ERR_INVALID_ARG;
      }
    if (!cfg.has_future_menu) break;
  }
  build_hands(g, set);
  for (int p = 0; p < 2; p++)
    if (g.n[p] == 0) {
      msg = "player " + std::to_string(p) + " has an empty range";
      return DCFR_ERR_EMPTY_RANGE;
    }
  if (!(g.num_combinations > 0.0)) {
    msg = "player 0 has an empty range";
    return DCFR_ERR_EMPTY_RANGE;
  }
  g.norm = 1.0 / g.num_combinations;
  g.half_pot = (double)cfg.root.pot / 2.0;
  build_iso(g);

  Ctx cx;
  cx.g = &g;
  cx.menu = &cfg.menu;
  cx.future = cfg.has_future_menu ? &cfg.future_menu : &cfg.menu;
  cx.root_street = cfg.root.street;
  cx.bb = cfg.big_blind;
  Betting root;
  root.street = cfg.root.street;
  root.pot = cfg.root.pot;
  for (int p = 0; p < 2; p++) {
    root.commit[p] = cfg.root.commit[p];
    root.stack[p] = cfg.root.stack[p];
    root.needs[p] = cfg.root.needs[p] != 0;
  }
  root.current_bet = cfg.root.current_bet;
  root.last_raise_inc = cfg.root.last_raise_inc;
  root.num_raises = cfg.root.num_raises;
  root.to_act = cfg.root.to_act;
  std::vector<int> dealt;
  g.stats = Stats();
  // The count draws from its own generator seeded 0 (count_tree,
  // tree.rs:338-343); the tree itself from one seeded with the configured
  // seed (Builder::new, tree.rs:415-420).
  StdRng count_rng(0);
  cx.rng = &count_rng;
  count_player(cx, root, dealt, g.stats);
  // StorageMode (storage.rs:79-85, lib.rs:346-352).
  uint64_t f32_bytes = reference_memory_bytes(g.stats, false);
  g.compressed = cfg.storage == DCFR_STORAGE_COMPRESSED || (cfg.storage == DCFR_STORAGE_AUTO && f32_bytes > (1ull << 30));
  if (!build_tree) return DCFR_OK;
  uint64_t needed = reference_memory_bytes(g.stats, g.compressed);
  if (needed > cfg.max_memory_bytes) {
    char buf[160];
    snprintf(buf, sizeof buf, "game tree needs ~%.2f GB but the limit is %.2f GB", (double)needed / 1e9,
             (double)cfg.max_memory_bytes / 1e9);
    msg = buf;
    return DCFR_ERR_TOO_LARGE;
  }
  g.nodes.clear();
  // The count gives the node total: one allocation, no regrowth copies.
  g.nodes.reserve((size_t)(g.stats.player + g.stats.chance + g.stats.terminal) + 1);
  g.chance.clear();
  g.boards.clear();
  g.storage_len = 0;
  g.player_nodes = 0;
  g.nodes.push_back(GNode());
  StdRng build_rng(cfg.chance_seed);
  cx.rng = &build_rng;
  fill_player(cx, 0, root, 0, 0, dealt);
  return DCFR_OK;
}

}  // namespace dcfr
