// TEST INFRASTRUCTURE — CPU oracle (see solver.hpp). Restates
// crates/solver/src/{tree,hands,iso,storage,cfr,river,eval,lib}.rs of
// AhanDatta/Poker-Trainer; each function cites the Rust it follows.
#include "solver.hpp"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <unordered_map>

namespace oracle {

static int g_threads = 0;
void set_num_threads(int n) { g_threads = n; }
int get_num_threads() { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

// Runs f inside one OpenMP parallel region (tasks spawned by chance nodes
// are executed by the team), or directly when already inside one.
template <class F>
static void par_region(F&& f) {
  int nt = get_num_threads();
  if (omp_in_parallel() || nt <= 1) {
    f();
    return;
  }
#pragma omp parallel num_threads(nt)
  {
#pragma omp single
    f();
  }
}

// ---------------------------------------------------------------- Discount
// cfr.rs:86-106.
Discount Discount::make(uint32_t t, const DcfrParams& params) {
  uint32_t tm = t < 1 ? 1 : t;
  double prev = (double)(tm - 1);
  double pa = std::pow(prev, params.alpha);
  double tf = (double)tm;
  float neg;
  if (!params.beta_clip) {
    double pb = std::pow(prev, params.beta);
    neg = (float)(pb / (pb + 1.0));
  } else {
    neg = 0.0f;
  }
  double since = tf - 1.0;
  if (params.restart_average) {
    uint32_t t0 = tm - 1;
    uint32_t p4 = t0 == 0 ? 0 : (1u << ((31u - (uint32_t)__builtin_clz(t0)) & ~1u));
    since = (double)(t0 - p4);
  }
  float strat = (float)std::pow(since / (since + 1.0), params.gamma);
  return Discount{(float)(pa / (pa + 1.0)), neg, strat, !params.unweighted_average};
}

// ---------------------------------------------------------------- betting
// tree.rs:49-61.
BettingState BettingState::street_start(Street s, Chips pot, Chips s0, Chips s1, Chips big_blind) {
  BettingState b;
  b.street = s;
  b.pot = pot;
  b.commit[0] = b.commit[1] = 0;
  b.stack[0] = s0;
  b.stack[1] = s1;
  b.current_bet = 0;
  b.last_raise_inc = big_blind;
  b.num_raises = 0;
  b.to_act = 0;
  b.needs[0] = s0 > 0;
  b.needs[1] = s1 > 0;
  return b;
}

// tree.rs:63-77.
Situation BettingState::situation(Chips big_blind) const {
  int p = to_act, o = p ^ 1;
  Situation s;
  s.street = street;
  s.pot = pot;
  s.to_call = std::min(std::max(current_bet - commit[p], (Chips)0), stack[p]);
  s.current_bet = current_bet;
  s.max_to = std::min(commit[p] + stack[p], commit[o] + stack[o]);
  s.min_raise_to = current_bet + std::max(last_raise_inc, big_blind);
  s.num_raises = num_raises;
  s.big_blind = big_blind;
  return s;
}

// tree.rs:93-125.
TransitionKind BettingState::apply(const Action& a, BettingState& s, Chips& put, int& folder) const {
  int p = to_act, o = p ^ 1;
  s = *this;
  put = 0;
  switch (a.kind) {
    case FOLD:
      folder = p;
      return T_FOLD;
    case CHECK: break;
    case CALL: put = std::min(std::max(s.current_bet - s.commit[p], (Chips)0), s.stack[p]); break;
    case RAISE: {
      put = a.amount - s.commit[p];
      Chips inc = a.amount - s.current_bet;
      if (inc >= s.last_raise_inc) s.last_raise_inc = inc;
      s.current_bet = a.amount;
      s.num_raises += 1;
      s.needs[o] = s.stack[o] > 0;
      break;
    }
  }
  s.commit[p] += put;
  s.stack[p] -= put;
  s.pot += put;
  s.needs[p] = false;
  if (s.needs[o]) {
    s.to_act = o;
    return T_CONTINUE;
  }
  return T_STREET_OVER;
}

std::vector<Action> Tree::actions(size_t id) const {
  std::vector<Action> out;
  const Node& n = nodes[id];
  for (uint32_t c = n.first_child; c < n.first_child + n.num_children; c++) out.push_back(nodes[c].edge_action);
  return out;
}

// ---------------------------------------------------------------- iso
const uint8_t ISO_PAIRS[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

int iso_pair_index(int a, int b) {
  if (a > b) std::swap(a, b);
  for (int i = 0; i < 6; i++)
    if (ISO_PAIRS[i][0] == a && ISO_PAIRS[i][1] == b) return i;
  return -1;
}

// iso.rs:25-36.
int swap_card(int card, int a, int b) {
  int s = card_suit(card);
  int s2 = s == a ? b : s == b ? a : s;
  return make_card(card_rank(card), s2);
}

static void suit_ranks(const std::vector<int>& board, uint16_t m[4]) {
  m[0] = m[1] = m[2] = m[3] = 0;
  for (int c : board) m[card_suit(c)] |= (uint16_t)(1u << card_rank(c));
}

// iso.rs:47-51.
std::vector<std::pair<int, int>> board_symmetric_pairs(const std::vector<int>& board) {
  uint16_t m[4];
  suit_ranks(board, m);
  std::vector<std::pair<int, int>> out;
  for (auto& pr : ISO_PAIRS)
    if (m[pr[0]] == m[pr[1]]) out.push_back({pr[0], pr[1]});
  return out;
}

// iso.rs:55-70.
std::vector<int> iso_orbit(const std::vector<int>& board, int combo) {
  auto pairs = board_symmetric_pairs(board);
  std::vector<int> orbit{combo};
  for (size_t i = 0; i < orbit.size(); i++) {
    const ComboCards& cc = combos_table()[orbit[i]];
    for (auto& pr : pairs) {
      int c = combo_index(swap_card(cc.hi, pr.first, pr.second), swap_card(cc.lo, pr.first, pr.second));
      if (std::find(orbit.begin(), orbit.end(), c) == orbit.end()) orbit.push_back(c);
    }
  }
  return orbit;
}

// iso.rs:89-116.
void Isomorphism::build(const HandSet& hands, bool en) {
  enabled = en;
  for (int i = 0; i < 6; i++) {
    range_symmetric[i] = false;
    perm[0][i].clear();
    perm[1][i].clear();
  }
  if (!en) return;
  for (int pi = 0; pi < 6; pi++) {
    int a = ISO_PAIRS[pi][0], b = ISO_PAIRS[pi][1];
    std::vector<uint16_t> pp[2];
    bool ok = true;
    for (int p = 0; p < 2 && ok; p++) {
      const std::vector<float>& w = hands.weights[p];
      float max_w = 0.0f;
      for (float x : w) max_w = std::max(max_w, x);
      max_w = std::max(max_w, 1e-30f);
      for (size_t h = 0; h < hands.cards[p].size(); h++) {
        int s1 = swap_card(hands.cards[p][h].first, a, b);
        int s2 = swap_card(hands.cards[p][h].second, a, b);
        uint32_t j = hands.lookup[p][combo_index(s1, s2)];
        if (j == NONE) {
          ok = false;
          break;
        }
        if (std::fabs(w[h] - w[j]) > 1e-4f * max_w) {
          ok = false;
          break;
        }
        pp[p].push_back((uint16_t)j);
      }
    }
    if (!ok) continue;
    range_symmetric[pi] = true;
    perm[0][pi] = pp[0];
    perm[1][pi] = pp[1];
  }
}

// iso.rs:120-141.
void Isomorphism::chance_cards(const std::vector<int>& board, const std::vector<int>& available,
                               std::vector<int>& canonical, std::vector<IsoRef>& refs) const {
  canonical.clear();
  refs.clear();
  bool any = false;
  for (int i = 0; i < 6; i++) any |= range_symmetric[i];
  if (!enabled || !any) {
    canonical = available;
    return;
  }
  uint16_t m[4];
  suit_ranks(board, m);
  for (int c : available) {
    int s = card_suit(c);
    int found = -1;
    for (int s0 = 0; s0 < s; s0++) {
      int pi = iso_pair_index(s0, s);
      if (range_symmetric[pi] && m[s0] == m[s]) {
        found = s0;
        break;
      }
    }
    if (found >= 0)
      refs.push_back(IsoRef{c, make_card(card_rank(c), found), iso_pair_index(found, s)});
    else
      canonical.push_back(c);
  }
}

// ---------------------------------------------------------------- hands
// hands.rs:35-76.
void HandSet::build(const std::vector<float> ranges[2], uint64_t board, float prune, const std::vector<int> keep[2]) {
  for (int p = 0; p < 2; p++) {
    combos[p].clear();
    cards[p].clear();
    weights[p].clear();
    float max_w = 0.0f;
    for (float x : ranges[p]) max_w = std::max(max_w, x);
    float cutoff = max_w * prune;
    for (int c = 0; c < 1326; c++) {
      const ComboCards& cc = combos_table()[c];
      if ((board >> cc.hi & 1) || (board >> cc.lo & 1)) continue;
      float w = ranges[p][c];
      bool forced = std::find(keep[p].begin(), keep[p].end(), c) != keep[p].end();
      if ((w > 0.0f && w >= cutoff) || (forced && w > 0.0f)) {
        combos[p].push_back((uint16_t)c);
        cards[p].push_back({cc.hi, cc.lo});
        weights[p].push_back(w);
      }
    }
  }
  for (int p = 0; p < 2; p++) {
    lookup[p].assign(1326, NONE);
    for (size_t i = 0; i < combos[p].size(); i++) lookup[p][combos[p][i]] = (uint32_t)i;
  }
  same[0].clear();
  same[1].clear();
  for (uint16_t c : combos[0]) same[0].push_back(lookup[1][c]);
  for (uint16_t c : combos[1]) same[1].push_back(lookup[0][c]);
  for (int p = 0; p < 2; p++) {
    blocked[p].assign(52, {});
    for (size_t i = 0; i < cards[p].size(); i++) {
      blocked[p][cards[p][i].first].push_back((uint32_t)i);
      blocked[p][cards[p][i].second].push_back((uint32_t)i);
    }
  }
  // compatible_weight (hands.rs:95-98).
  std::vector<double> compat = compatible_reach(0, weights[1].data());
  double s = -0.0;
  for (size_t i = 0; i < compat.size(); i++) s += compat[i] * (double)weights[0][i];
  num_combinations = s;
}

// hands.rs:102-125.
std::vector<double> HandSet::compatible_reach(int p, const float* opp_reach) const {
  int o = p ^ 1;
  double total = 0.0;
  double minus[52] = {0};
  for (size_t k = 0; k < cards[o].size(); k++) {
    float w = opp_reach[k];
    if (w != 0.0f) {
      double wd = (double)w;
      total += wd;
      minus[cards[o][k].first] += wd;
      minus[cards[o][k].second] += wd;
    }
  }
  std::vector<double> out(cards[p].size());
  for (size_t i = 0; i < cards[p].size(); i++) {
    double s = same[p][i] == NONE ? 0.0 : (double)opp_reach[same[p][i]];
    double v = total - minus[cards[p][i].first] - minus[cards[p][i].second] + s;
    out[i] = v > 0.0 ? v : 0.0;
  }
  return out;
}

// hands.rs:137-158.
void StrengthTable::build(const HandSet& hands, const std::vector<int>& board) {
  uint64_t mask = 0, bset = 0;
  for (int c : board) {
    mask |= eval_card_bit(c);
    bset |= 1ull << c;
  }
  for (int p = 0; p < 2; p++) {
    lists[p].clear();
    for (size_t i = 0; i < hands.cards[p].size(); i++) {
      int a = hands.cards[p][i].first, b = hands.cards[p][i].second;
      if ((bset >> a & 1) || (bset >> b & 1)) continue;
      lists[p].push_back(Entry{evaluate_mask(mask | eval_card_bit(a) | eval_card_bit(b)), (uint16_t)i, (uint8_t)a,
                               (uint8_t)b});
    }
    std::sort(lists[p].begin(), lists[p].end(), [](const Entry& x, const Entry& y) {
      if (x.strength != y.strength) return x.strength < y.strength;
      if (x.idx != y.idx) return x.idx < y.idx;
      if (x.c1 != y.c1) return x.c1 < y.c1;
      return x.c2 < y.c2;
    });
  }
}

// ---------------------------------------------------------------- sampling
static inline uint32_t rotl32(uint32_t v, int n) { return (v << n) | (v >> (32 - n)); }

void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]) {
  // "expand 32-byte k"
  const uint32_t init[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u,
                             key[0], key[1], key[2], key[3], key[4], key[5], key[6], key[7],
                             (uint32_t)(counter & 0xffffffffu), (uint32_t)(counter >> 32),
                             (uint32_t)(stream & 0xffffffffu), (uint32_t)(stream >> 32)};
  uint32_t x[16];
  std::memcpy(x, init, sizeof x);
  auto qr = [&x](int a, int b, int c, int d) {
    x[a] += x[b];
    x[d] ^= x[a];
    x[d] = rotl32(x[d], 16);
    x[c] += x[d];
    x[b] ^= x[c];
    x[b] = rotl32(x[b], 12);
    x[a] += x[b];
    x[d] ^= x[a];
    x[d] = rotl32(x[d], 8);
    x[c] += x[d];
    x[b] ^= x[c];
    x[b] = rotl32(x[b], 7);
  };
  for (int i = 0; i < rounds / 2; i++) {
    // column round, then diagonal round
    qr(0, 4, 8, 12);
    qr(1, 5, 9, 13);
    qr(2, 6, 10, 14);
    qr(3, 7, 11, 15);
    qr(0, 5, 10, 15);
    qr(1, 6, 11, 12);
    qr(2, 7, 8, 13);
    qr(3, 4, 9, 14);
  }
  for (int i = 0; i < 16; i++) out[i] = x[i] + init[i];
}

ChaChaRng::ChaChaRng(uint64_t state) {
  // seed_from_u64: eight PCG32 steps, each output one little-endian key word.
  const uint64_t MUL = 6364136223846793005ull, INC = 11634580027462260723ull;
  for (int i = 0; i < 8; i++) {
    state = state * MUL + INC;
    uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
    uint32_t rot = (uint32_t)(state >> 59);
    key[i] = rot == 0 ? xorshifted : (xorshifted >> rot) | (xorshifted << (32 - rot));
  }
}

uint64_t ChaChaRng::next_u64() {
  // BlockRng::next_u64: two words, low first; a pair that straddles the
  // buffer end takes the last word and the first of the next buffer.
  auto generate = [this]() {
    for (int b = 0; b < 4; b++) chacha_block(key, block_counter + (uint64_t)b, 0, 12, results + 16 * b);
    block_counter += 4;
  };
  if (index < 63) {
    uint64_t v = (uint64_t)results[index] | ((uint64_t)results[index + 1] << 32);
    index += 2;
    return v;
  }
  if (index >= 64) {
    generate();
    index = 2;
    return (uint64_t)results[0] | ((uint64_t)results[1] << 32);
  }
  uint64_t lo = results[63];
  generate();
  index = 1;
  return lo | ((uint64_t)results[0] << 32);
}

double ChaChaRng::random_f64() {
  const double scale = 1.0 / (double)(1ull << 53);
  return scale * (double)(next_u64() >> (64 - 53));
}

std::vector<int> sample_cards(const std::vector<int>& available, size_t k, ChaChaRng& rng) {
  if (k >= available.size()) return available;
  std::vector<int> by_suit[4];
  for (int c : available) by_suit[card_suit(c)].push_back(c);
  for (auto& v : by_suit)
    std::sort(v.begin(), v.end(), [](int a, int b) { return card_rank(a) < card_rank(b); });
  double total = (double)available.size();
  size_t quotas[4] = {0, 0, 0, 0};
  std::vector<std::tuple<double, double, size_t>> fracs;
  for (size_t s = 0; s < 4; s++) {
    double exact = (double)k * (double)by_suit[s].size() / total;
    quotas[s] = (size_t)std::floor(exact);
    fracs.emplace_back(exact - std::floor(exact), rng.random_f64(), s);
  }
  size_t assigned = quotas[0] + quotas[1] + quotas[2] + quotas[3];
  std::sort(fracs.begin(), fracs.end(), [](const auto& a, const auto& b) { return b < a; });
  for (auto& f : fracs) {
    if (assigned >= k) break;
    size_t s = std::get<2>(f);
    if (quotas[s] < by_suit[s].size()) {
      quotas[s] += 1;
      assigned += 1;
    }
  }
  std::vector<int> out;
  for (size_t s = 0; s < 4; s++) {
    size_t m = by_suit[s].size(), q = quotas[s];
    if (q == 0) continue;
    double step = (double)m / (double)q;
    double offset = rng.random_f64() * step;
    for (size_t j = 0; j < q; j++) {
      size_t idx = std::min((size_t)std::floor(offset + (double)j * step), m - 1);
      out.push_back(by_suit[s][idx]);
    }
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

// ---------------------------------------------------------------- tree
struct TreeParams {
  Street root_street;
  const std::vector<int>* root_board;
  const PostflopMenu* menu;
  const PostflopMenu* future_menu;
  Chips big_blind;
  size_t num_hands[2];
  double rake_rate, rake_cap;
  const Isomorphism* iso;
  bool sampled = false;
  size_t sample_turn = 0, sample_river = 0;
  ChaChaRng* rng = nullptr;  // the builder's (or the count's) generator

  const PostflopMenu& menu_for(Street s) const { return s == root_street ? *menu : *future_menu; }
  std::vector<Action> actions(const BettingState& st) const {
    return postflop_actions(st.situation(big_blind), menu_for(st.street));
  }
  // tree.rs:310-312.
  float rake(Chips pot) const { return (float)std::min((double)pot * rake_rate, rake_cap); }
  // tree.rs:302-308.
  size_t sample_size(Street next, bool& has) const {
    has = sampled;
    return next == TURN ? sample_turn : sample_river;
  }
  // tree.rs:315-334.
  void chance_cards(const std::vector<int>& dealt, bool all_in, Street next, std::vector<int>& canon,
                    std::vector<IsoRef>& refs, size_t& n_avail) const {
    std::vector<int> board = *root_board;
    board.insert(board.end(), dealt.begin(), dealt.end());
    uint64_t used = 0;
    for (int c : board) used |= 1ull << c;
    std::vector<int> available;
    for (int c = 0; c < 52; c++)
      if (!(used >> c & 1)) available.push_back(c);
    n_avail = available.size();
    bool has;
    size_t k = sample_size(next, has);
    if (!all_in && has && k < n_avail) {
      canon = sample_cards(available, k, *rng);
      refs.clear();
      return;
    }
    iso->chance_cards(board, available, canon, refs);
  }
};

static void count_after_street(const TreeParams& params, const BettingState& st, std::vector<int>& dealt,
                               TreeStats& stats);

// tree.rs:345-362.
static void count_player(const TreeParams& params, const BettingState& st, std::vector<int>& dealt, TreeStats& stats) {
  stats.player_nodes += 1;
  auto actions = params.actions(st);
  stats.storage_cells += (uint64_t)(actions.size() * params.num_hands[st.to_act]);
  for (auto& a : actions) {
    BettingState s2;
    Chips put;
    int f;
    switch (st.apply(a, s2, put, f)) {
      case T_CONTINUE: count_player(params, s2, dealt, stats); break;
      case T_FOLD: stats.terminal_nodes += 1; break;
      case T_STREET_OVER: count_after_street(params, s2, dealt, stats); break;
    }
  }
}

// tree.rs:364-401.
static void count_after_street(const TreeParams& params, const BettingState& st, std::vector<int>& dealt,
                               TreeStats& stats) {
  if (st.street == RIVER) {
    stats.terminal_nodes += 1;
    return;
  }
  stats.chance_nodes += 1;
  bool all_in = st.stack[0] == 0 || st.stack[1] == 0;
  Street next = (Street)(st.street + 1);
  std::vector<int> cards;
  std::vector<IsoRef> refs;
  size_t n_avail;
  params.chance_cards(dealt, all_in, next, cards, refs, n_avail);
  bool uniform = refs.empty() && !params.iso->enabled;
  size_t nreps = uniform ? 1 : cards.size();
  TreeStats sub;
  for (size_t i = 0; i < nreps; i++) {
    dealt.push_back(cards[i]);
    if (all_in) {
      BettingState s2 = st;
      s2.street = next;
      count_after_street(params, s2, dealt, sub);
    } else {
      BettingState s2 = BettingState::street_start(next, st.pot, st.stack[0], st.stack[1], params.big_blind);
      count_player(params, s2, dealt, sub);
    }
    dealt.pop_back();
  }
  uint64_t k = uniform ? (uint64_t)cards.size() : 1;
  stats.player_nodes += sub.player_nodes * k;
  stats.chance_nodes += sub.chance_nodes * k;
  stats.terminal_nodes += sub.terminal_nodes * k;
  stats.storage_cells += sub.storage_cells * k;
}

// Builder (tree.rs:404-573).
struct Builder {
  const TreeParams& params;
  Tree tree;
  std::unordered_map<uint64_t, uint32_t> board_index;

  explicit Builder(const TreeParams& p) : params(p) {}

  size_t alloc_children(size_t k) {
    size_t first = tree.nodes.size();
    tree.nodes.resize(first + k, Node());
    return first;
  }

  void build(const BettingState& root) {
    tree.nodes.push_back(Node());
    std::vector<int> dealt;
    fill_player(0, root, 0, 0, dealt);
  }

  void fill_player(size_t id, const BettingState& st, int32_t inv0, int32_t inv1, std::vector<int>& dealt) {
    auto actions = params.actions(st);
    size_t k = actions.size();
    size_t first = alloc_children(k);
    Node& n = tree.nodes[id];
    EdgeKind ek = n.edge_kind;
    Action ea = n.edge_action;
    int ec = n.edge_card;
    Node nn;
    nn.kind = K_PLAYER;
    nn.player = (uint8_t)st.to_act;
    nn.street = st.street;
    nn.num_children = (uint16_t)k;
    nn.first_child = (uint32_t)first;
    nn.invest[0] = inv0;
    nn.invest[1] = inv1;
    nn.offset = tree.storage_len;
    nn.slot = tree.num_player_nodes;
    nn.rake = 0.0f;
    nn.chance_factor = 1.0f;
    nn.edge_kind = ek;
    nn.edge_action = ea;
    nn.edge_card = ec;
    tree.nodes[id] = nn;
    tree.storage_len += (uint64_t)(k * params.num_hands[st.to_act]);
    tree.num_player_nodes += 1;
    for (size_t i = 0; i < k; i++) {
      size_t child = first + i;
      BettingState s2;
      Chips put;
      int f;
      TransitionKind tr = st.apply(actions[i], s2, put, f);
      int32_t inv[2] = {inv0, inv1};
      inv[st.to_act] += (int32_t)put;
      if (tr == T_CONTINUE) {
        tree.nodes[child].edge_kind = E_ACTION;
        tree.nodes[child].edge_action = actions[i];
        fill_player(child, s2, inv[0], inv[1], dealt);
      } else if (tr == T_FOLD) {
        int o = f ^ 1;
        Chips uncalled = std::max(st.commit[o] - st.commit[f], (Chips)0);
        Node t;
        t.kind = K_FOLD;
        t.player = (uint8_t)f;
        t.street = st.street;
        t.invest[0] = inv[0];
        t.invest[1] = inv[1];
        t.rake = params.rake(st.pot - uncalled);
        t.edge_kind = E_ACTION;
        t.edge_action = actions[i];
        tree.nodes[child] = t;
      } else {
        tree.nodes[child].edge_kind = E_ACTION;
        tree.nodes[child].edge_action = actions[i];
        fill_after_street(child, s2, inv[0], inv[1], dealt);
      }
    }
  }

  void fill_after_street(size_t id, const BettingState& st, int32_t inv0, int32_t inv1, std::vector<int>& dealt) {
    EdgeKind ek = tree.nodes[id].edge_kind;
    Action ea = tree.nodes[id].edge_action;
    int ec = tree.nodes[id].edge_card;
    if (st.street == RIVER) {
      uint32_t table = table_for(dealt);
      Node n;
      n.kind = K_SHOWDOWN;
      n.street = RIVER;
      n.invest[0] = inv0;
      n.invest[1] = inv1;
      n.offset = table;
      n.rake = params.rake(st.pot);
      n.edge_kind = ek;
      n.edge_action = ea;
      n.edge_card = ec;
      tree.nodes[id] = n;
      return;
    }
    bool all_in = st.stack[0] == 0 || st.stack[1] == 0;
    Street next = (Street)(st.street + 1);
    std::vector<int> cards;
    std::vector<IsoRef> refs;
    size_t n_avail;
    params.chance_cards(dealt, all_in, next, cards, refs, n_avail);
    size_t board_len = params.root_board->size() + dealt.size();
    float compatible = (float)(52 - board_len - 4);
    size_t total_cards = cards.size() + refs.size();
    size_t first = alloc_children(cards.size());
    uint32_t slot = (uint32_t)tree.chance.size();
    ChanceInfo info;
    for (auto& r : refs) {
      size_t k = std::find(cards.begin(), cards.end(), r.canonical) - cards.begin();
      info.iso.push_back({(uint16_t)k, (uint8_t)r.pair});
      info.iso_cards.push_back(r.card);
    }
    tree.chance.push_back(info);
    Node n;
    n.kind = K_CHANCE;
    n.street = st.street;
    n.num_children = (uint16_t)cards.size();
    n.first_child = (uint32_t)first;
    n.invest[0] = inv0;
    n.invest[1] = inv1;
    n.slot = slot;
    // tree.rs:542: all f32 arithmetic.
    float tc = (float)total_cards;
    float na = (float)n_avail;
    float denom = tc * compatible / na;
    n.chance_factor = 1.0f / denom;
    n.edge_kind = ek;
    n.edge_action = ea;
    n.edge_card = ec;
    tree.nodes[id] = n;
    for (size_t i = 0; i < cards.size(); i++) {
      size_t child = first + i;
      tree.nodes[child].edge_kind = E_CARD;
      tree.nodes[child].edge_card = cards[i];
      dealt.push_back(cards[i]);
      if (all_in) {
        BettingState s2 = st;
        s2.street = next;
        fill_after_street(child, s2, inv0, inv1, dealt);
      } else {
        BettingState s2 = BettingState::street_start(next, st.pot, st.stack[0], st.stack[1], params.big_blind);
        fill_player(child, s2, inv0, inv1, dealt);
      }
      dealt.pop_back();
    }
  }

  uint32_t table_for(const std::vector<int>& dealt) {
    uint64_t key = 0;
    for (int c : dealt) key |= 1ull << c;
    auto it = board_index.find(key);
    if (it != board_index.end()) return it->second;
    uint32_t i = (uint32_t)tree.boards.size();
    std::vector<int> board = *params.root_board;
    board.insert(board.end(), dealt.begin(), dealt.end());
    tree.boards.push_back(board);
    board_index[key] = i;
    return i;
  }
};

// ---------------------------------------------------------------- scratch
// Thread-local pool of f32 buffers (scratch.rs:7-50).
struct Buf {
  std::vector<float> v;
  static std::vector<std::vector<float>>& pool() {
    static thread_local std::vector<std::vector<float>> p;
    return p;
  }
  explicit Buf(size_t n) {
    auto& p = pool();
    if (!p.empty()) {
      v = std::move(p.back());
      p.pop_back();
    }
    v.resize(n);
  }
  Buf(const float* src, size_t n) : Buf(n) { std::memcpy(v.data(), src, n * sizeof(float)); }
  ~Buf() { pool().push_back(std::move(v)); }
  float* data() { return v.data(); }
  float& operator[](size_t i) { return v[i]; }
  size_t size() const { return v.size(); }
};

// ---------------------------------------------------------------- cfr
struct Ctx {
  const Tree* tree;
  Storage* store;
  const HandSet* hands;
  const std::vector<StrengthTable>* tables;
  const Isomorphism* iso;
  double half_pot;
  double norm;
  bool batch_river;
};

// cfr.rs:114-121.
static inline float recip(float d) {
  float i = 1.0f / d;
  return (d > 0.0f && std::isfinite(i)) ? i : 0.0f;
}

static inline float fmax0(float x) { return x > 0.0f ? x : 0.0f; }

// cfr.rs:124-154.
static void normalize_in_place(float* s, size_t na, size_t n) {
  if (n == 0) return;
  Buf inv(s, n);
  for (size_t a = 1; a < na; a++)
    for (size_t h = 0; h < n; h++) inv[h] += s[a * n + h];
  bool any_zero = false;
  for (size_t h = 0; h < n; h++) {
    inv[h] = recip(inv[h]);
    any_zero |= inv[h] == 0.0f;
  }
  for (size_t a = 0; a < na; a++)
    for (size_t h = 0; h < n; h++) s[a * n + h] *= inv[h];
  if (any_zero) {
    float uniform = 1.0f / (float)na;
    for (size_t h = 0; h < n; h++)
      if (inv[h] == 0.0f)
        for (size_t a = 0; a < na; a++) s[a * n + h] = uniform;
  }
}

// cfr.rs:196-207.
// Regrets as f32: stored f32, or undecoded i16 (regret matching is
// invariant under the node's positive scale; cfr.rs:155-160).
static inline float as_f32(float x) { return x; }
static inline float as_f32(int16_t x) { return (float)x; }

template <class T>
static void positive_sums(const T* r, size_t na, size_t n, float* sums) {
  for (size_t h = 0; h < n; h++) sums[h] = fmax0(as_f32(r[h]));
  for (size_t a = 1; a < na; a++)
    for (size_t h = 0; h < n; h++) sums[h] += fmax0(as_f32(r[a * n + h]));
}

// cfr.rs:161-192.
template <class T>
static void regret_match_into(const T* r, size_t na, size_t n, float* out) {
  if (n == 0) return;
  Buf inv(n);
  positive_sums(r, na, n, inv.data());
  bool any_zero = false;
  for (size_t h = 0; h < n; h++) {
    inv[h] = recip(inv[h]);
    any_zero |= inv[h] == 0.0f;
  }
  for (size_t a = 0; a < na; a++)
    for (size_t h = 0; h < n; h++) out[a * n + h] = fmax0(as_f32(r[a * n + h])) * inv[h];
  if (any_zero) {
    float uniform = 1.0f / (float)na;
    for (size_t h = 0; h < n; h++)
      if (inv[h] == 0.0f)
        for (size_t a = 0; a < na; a++) out[a * n + h] = uniform;
  }
}

// ---- Storage accessors (storage.rs:226-330) ----
// max(|x|) over a block (storage.rs:113-128; a max is order-free).
static float max_abs(const float* v, size_t len) {
  float m = 0.0f;
  for (size_t i = 0; i < len; i++) m = std::fmax(m, std::fabs(v[i]));
  return m;
}

// load_current_strategy (storage.rs:244-255).
static void load_current_strategy(const Storage& st, const Node& node, size_t n, float* out) {
  const size_t na = node.num_children;
  if (st.compressed) regret_match_into(st.rq.data() + node.offset, na, n, out);
  else regret_match_into(st.regrets.data() + node.offset, na, n, out);
}

// load_strat (storage.rs:256-268).
static void load_strat(const Storage& st, const Node& node, size_t n, float* out) {
  const size_t len = node.num_children * n;
  if (!st.compressed) {
    std::memcpy(out, st.strat.data() + node.offset, len * sizeof(float));
    return;
  }
  const float scale = st.sscale[node.slot] / 65535.0f;
  const uint16_t* q = st.sq.data() + node.offset;
  for (size_t i = 0; i < len; i++) out[i] = (float)q[i] * scale;
}

// update_regrets (storage.rs:272-303): f on the decoded regrets, then the
// node's new scale max|r| and round half away from zero, saturating.
template <class F>
static void update_regrets(Storage& st, const Node& node, size_t n, F f) {
  const size_t len = node.num_children * n;
  if (!st.compressed) {
    f(st.regrets.data() + node.offset);
    return;
  }
  Buf buf(len);
  float& scale_slot = st.rscale[node.slot];
  int16_t* q = st.rq.data() + node.offset;
  const float scale = scale_slot / 32767.0f;
  for (size_t i = 0; i < len; i++) buf[i] = (float)q[i] * scale;
  f(buf.data());
  const float mx = max_abs(buf.data(), len);
  scale_slot = mx;
  if (mx > 0.0f) {
    const float inv = 32767.0f / mx;
    for (size_t i = 0; i < len; i++) {
      const float y = buf[i] * inv;
      const float t = y + std::copysign(0.5f, y);
      // Rust's `as i16`: truncation toward zero, saturating, NaN to 0.
      q[i] = t != t ? (int16_t)0 : t >= 32767.0f ? (int16_t)32767 : t <= -32768.0f ? (int16_t)-32768 : (int16_t)t;
    }
  } else {
    std::fill(q, q + len, (int16_t)0);
  }
}

// update_strat (storage.rs:306-330): values kept non-negative, u16 with the
// node's max, rounded half up.
template <class F>
static void update_strat(Storage& st, const Node& node, size_t n, F f) {
  const size_t len = node.num_children * n;
  if (!st.compressed) {
    f(st.strat.data() + node.offset);
    return;
  }
  Buf buf(len);
  float& scale_slot = st.sscale[node.slot];
  uint16_t* q = st.sq.data() + node.offset;
  const float scale = scale_slot / 65535.0f;
  for (size_t i = 0; i < len; i++) buf[i] = (float)q[i] * scale;
  f(buf.data());
  const float mx = max_abs(buf.data(), len);
  scale_slot = mx;
  if (mx > 0.0f) {
    const float inv = 65535.0f / mx;
    for (size_t i = 0; i < len; i++) {
      const float t = std::fmax(buf[i], 0.0f) * inv + 0.5f;
      q[i] = t != t ? (uint16_t)0 : t >= 65535.0f ? (uint16_t)65535 : (uint16_t)t;
    }
  } else {
    std::fill(q, q + len, (uint16_t)0);
  }
}

// cfr.rs:226-235.
static double fold_payoff(const Ctx& ctx, const Node& node, int p) {
  int f = node.player;
  double v;
  if (f == p)
    v = -(ctx.half_pot + (double)node.invest[p]);
  else
    v = ctx.half_pot + (double)node.invest[f] - (double)node.rake;
  return v * ctx.norm;
}

// cfr.rs:239-246.
static void showdown_payoffs(const Ctx& ctx, const Node& node, int p, double& win, double& lose, double& tie) {
  int o = p ^ 1;
  double rake = (double)node.rake;
  win = (ctx.half_pot + (double)node.invest[o] - rake) * ctx.norm;
  lose = -(ctx.half_pot + (double)node.invest[p]) * ctx.norm;
  tie = 0.5 * ((double)(node.invest[o] - node.invest[p]) - rake) * ctx.norm;
}

// ---------------------------------------------------------------- eval
// eval.rs:20-37.
static inline void accumulate(uint8_t c1, uint8_t c2, float w, double& sum, double* minus) {
  if (w != 0.0f) {
    double wd = (double)w;
    sum += wd;
    minus[c1] += wd;
    minus[c2] += wd;
  }
}

// eval.rs:40-64.
void eval_fold(const HandSet& hs, int p, const float* opp_reach, double payoff, float* out) {
  int o = p ^ 1;
  double total = 0.0;
  double minus[52] = {0};
  for (size_t k = 0; k < hs.cards[o].size(); k++)
    accumulate(hs.cards[o][k].first, hs.cards[o][k].second, opp_reach[k], total, minus);
  size_t n = hs.cards[p].size();
  if (total == 0.0) {
    for (size_t h = 0; h < n; h++) out[h] = 0.0f;
    return;
  }
  for (size_t h = 0; h < n; h++) {
    uint32_t sm = hs.same[p][h];
    double s = sm == NONE ? 0.0 : (double)opp_reach[sm];
    double m2 = minus[hs.cards[p][h].first] + minus[hs.cards[p][h].second];
    out[h] = (float)(payoff * (total - m2 + s));
  }
}

// eval.rs:347-379.
static void add_ties(const HandSet& hs, const StrengthTable& table, int p, const float* opp_reach, double tie,
                     float* out) {
  int o = p ^ 1;
  const auto& mine = table.lists[p];
  const auto& theirs = table.lists[o];
  size_t j = 0, k = 0;
  while (k < mine.size()) {
    uint32_t s = mine[k].strength;
    while (j < theirs.size() && theirs[j].strength < s) j++;
    double eq_sum = 0.0;
    double eq_minus[52] = {0};
    size_t jj = j;
    while (jj < theirs.size() && theirs[jj].strength == s) {
      const Entry& e = theirs[jj];
      accumulate(e.c1, e.c2, opp_reach[e.idx], eq_sum, eq_minus);
      jj++;
    }
    while (k < mine.size() && mine[k].strength == s) {
      const Entry& e = mine[k];
      size_t i = e.idx;
      double same_w = hs.same[p][i] == NONE ? 0.0 : (double)opp_reach[hs.same[p][i]];
      double eq = eq_sum - (eq_minus[e.c1] + eq_minus[e.c2]) + same_w;
      out[i] += (float)(tie * eq);
      k++;
    }
  }
}

// eval.rs:69-148.
void eval_showdown(const HandSet& hs, const StrengthTable& table, int p, const float* opp_reach, double win,
                   double lose, double tie, float* out) {
  int o = p ^ 1;
  size_t n = hs.cards[p].size();
  for (size_t h = 0; h < n; h++) out[h] = 0.0f;
  const auto& mine = table.lists[p];
  const auto& theirs = table.lists[o];
  double sum = 0.0;
  double minus[52] = {0};
  size_t j = 0, k = 0;
  while (k < mine.size()) {
    uint32_t s = mine[k].strength;
    while (j < theirs.size()) {
      const Entry& e = theirs[j];
      if (e.strength >= s) break;
      accumulate(e.c1, e.c2, opp_reach[e.idx], sum, minus);
      j++;
    }
    while (k < mine.size()) {
      const Entry& e = mine[k];
      if (e.strength != s) break;
      out[e.idx] = (float)(win * (sum - (minus[e.c1] + minus[e.c2])));
      k++;
    }
  }
  sum = 0.0;
  std::memset(minus, 0, sizeof(minus));
  j = theirs.size();
  k = mine.size();
  while (k > 0) {
    uint32_t s = mine[k - 1].strength;
    while (j > 0) {
      const Entry& e = theirs[j - 1];
      if (e.strength <= s) break;
      accumulate(e.c1, e.c2, opp_reach[e.idx], sum, minus);
      j--;
    }
    while (k > 0) {
      const Entry& e = mine[k - 1];
      if (e.strength != s) break;
      out[e.idx] += (float)(lose * (sum - (minus[e.c1] + minus[e.c2])));
      k--;
    }
  }
  if (tie != 0.0) add_ties(hs, table, p, opp_reach, tie, out);
}

constexpr size_t LANES = 4;  // eval.rs:151

// eval.rs:173-206.
void fold_batch(const HandSet& hs, int p, const std::vector<const float*>& reaches, const std::vector<double>& payoffs,
                const std::vector<float*>& outs) {
  size_t k = reaches.size();
  int o = p ^ 1;
  double total[LANES] = {0, 0, 0, 0};
  double minus[52][LANES];
  std::memset(minus, 0, sizeof(minus));
  for (size_t j = 0; j < hs.cards[o].size(); j++) {
    double w[LANES] = {0, 0, 0, 0};
    bool nz = false;
    for (size_t t = 0; t < k; t++) {
      w[t] = (double)reaches[t][j];
      nz |= w[t] != 0.0;
    }
    if (!nz) continue;
    int a = hs.cards[o][j].first, b = hs.cards[o][j].second;
    for (size_t t = 0; t < LANES; t++) {
      total[t] += w[t];
      minus[a][t] += w[t];
      minus[b][t] += w[t];
    }
  }
  for (size_t h = 0; h < hs.cards[p].size(); h++) {
    int a = hs.cards[p][h].first, b = hs.cards[p][h].second;
    uint32_t s = hs.same[p][h];
    for (size_t t = 0; t < k; t++) {
      double sw = s == NONE ? 0.0 : (double)reaches[t][s];
      outs[t][h] = (float)(payoffs[t] * (total[t] - minus[a][t] - minus[b][t] + sw));
    }
  }
}

// eval.rs:214-344. outs must be zero-initialized.
void showdown_batch(const HandSet& hs, const StrengthTable& table, int p, const std::vector<const float*>& reaches,
                    const std::vector<double>& win, const std::vector<double>& lose, const std::vector<double>& tie,
                    const std::vector<float*>& outs, const std::vector<std::pair<double, float*>>& folds,
                    const std::vector<bool>& has_fold) {
  size_t k = reaches.size();
  int o = p ^ 1;
  const auto& mine = table.lists[p];
  const auto& theirs = table.lists[o];
  double wv[LANES] = {0, 0, 0, 0}, lv[LANES] = {0, 0, 0, 0};
  for (size_t t = 0; t < k; t++) {
    wv[t] = win[t];
    lv[t] = lose[t];
  }
  static thread_local std::vector<double> inter, res;
  inter.assign(theirs.size() * LANES, 0.0);
  for (size_t j = 0; j < theirs.size(); j++)
    for (size_t t = 0; t < k; t++) inter[j * LANES + t] = (double)reaches[t][theirs[j].idx];
  res.assign(mine.size() * LANES, 0.0);
  auto nonzero = [&](size_t j) {
    for (size_t t = 0; t < LANES; t++)
      if (inter[j * LANES + t] != 0.0) return true;
    return false;
  };
  double sum[LANES] = {0, 0, 0, 0};
  double minus[52][LANES];
  std::memset(minus, 0, sizeof(minus));
  size_t i = 0, j = 0;
  while (i < mine.size()) {
    uint32_t s = mine[i].strength;
    while (j < theirs.size() && theirs[j].strength < s) {
      if (nonzero(j)) {
        const Entry& e = theirs[j];
        for (size_t t = 0; t < LANES; t++) {
          double w = inter[j * LANES + t];
          sum[t] += w;
          minus[e.c1][t] += w;
          minus[e.c2][t] += w;
        }
      }
      j++;
    }
    while (i < mine.size() && mine[i].strength == s) {
      const Entry& e = mine[i];
      for (size_t t = 0; t < LANES; t++) res[i * LANES + t] = wv[t] * (sum[t] - minus[e.c1][t] - minus[e.c2][t]);
      i++;
    }
  }
  bool any_fold = false;
  for (size_t t = 0; t < k; t++) any_fold |= has_fold[t];
  if (any_fold) {
    while (j < theirs.size()) {
      if (nonzero(j)) {
        const Entry& e = theirs[j];
        for (size_t t = 0; t < LANES; t++) {
          double w = inter[j * LANES + t];
          sum[t] += w;
          minus[e.c1][t] += w;
          minus[e.c2][t] += w;
        }
      }
      j++;
    }
    for (size_t t = 0; t < k; t++) {
      if (!has_fold[t]) continue;
      double pay = folds[t].first;
      float* out = folds[t].second;
      const float* reach = reaches[t];
      for (size_t h = 0; h < hs.cards[p].size(); h++) {
        uint32_t sm = hs.same[p][h];
        double sw = sm == NONE ? 0.0 : (double)reach[sm];
        int a = hs.cards[p][h].first, b = hs.cards[p][h].second;
        out[h] = (float)(pay * (sum[t] - minus[a][t] - minus[b][t] + sw));
      }
    }
  }
  double sum2[LANES] = {0, 0, 0, 0};
  std::memset(minus, 0, sizeof(minus));
  i = mine.size();
  j = theirs.size();
  while (i > 0) {
    uint32_t s = mine[i - 1].strength;
    while (j > 0 && theirs[j - 1].strength > s) {
      if (nonzero(j - 1)) {
        const Entry& e = theirs[j - 1];
        for (size_t t = 0; t < LANES; t++) {
          double w = inter[(j - 1) * LANES + t];
          sum2[t] += w;
          minus[e.c1][t] += w;
          minus[e.c2][t] += w;
        }
      }
      j--;
    }
    while (i > 0 && mine[i - 1].strength == s) {
      const Entry& e = mine[i - 1];
      for (size_t t = 0; t < LANES; t++)
        res[(i - 1) * LANES + t] += lv[t] * (sum2[t] - minus[e.c1][t] - minus[e.c2][t]);
      i--;
    }
  }
  for (size_t q = 0; q < mine.size(); q++)
    for (size_t t = 0; t < k; t++) outs[t][mine[q].idx] = (float)res[q * LANES + t];
  for (size_t t = 0; t < k; t++)
    if (tie[t] != 0.0) add_ties(hs, table, p, reaches[t], tie[t], outs[t]);
}

// ---------------------------------------------------------------- traversal
static void traverse(const Ctx& ctx, size_t id, int p, const float* opp_reach, size_t nq, const Mode& mode, float* out,
                     size_t n);

// own_node_update (cfr.rs:315-382).
static void own_node_update(const Ctx& ctx, const Node& node, size_t n, const float* cfv, const Mode& mode,
                            float* out) {
  size_t na = node.num_children;
  if (mode.kind == MODE_BR) {
    for (size_t h = 0; h < n; h++) out[h] = cfv[h];
    for (size_t a = 1; a < na; a++)
      for (size_t h = 0; h < n; h++) {
        float v = cfv[a * n + h];
        out[h] = v > out[h] ? v : out[h];
      }
  } else if (mode.kind == MODE_AVG) {
    Buf s(na * n);
    load_strat(*ctx.store, node, n, s.data());
    normalize_in_place(s.data(), na, n);
    for (size_t h = 0; h < n; h++) out[h] = 0.0f;
    for (size_t a = 0; a < na; a++)
      for (size_t h = 0; h < n; h++) out[h] += s[a * n + h] * cfv[a * n + h];
  } else {
    update_regrets(*ctx.store, node, n, [&](float* r) {
    const Discount& d = mode.d;
    Buf inv(n);
    positive_sums(r, na, n, inv.data());
    for (size_t h = 0; h < n; h++) out[h] = 0.0f;
    for (size_t a = 0; a < na; a++)
      for (size_t h = 0; h < n; h++) out[h] += fmax0(r[a * n + h]) * cfv[a * n + h];
    bool any_zero = false;
    for (size_t h = 0; h < n; h++) {
      inv[h] = recip(inv[h]);
      any_zero |= inv[h] == 0.0f;
      out[h] *= inv[h];
    }
    if (any_zero) {
      float mean = 1.0f / (float)na;
      for (size_t h = 0; h < n; h++)
        if (inv[h] == 0.0f) {
          float s = -0.0f;  // f32 Sum starts at -0.0
          for (size_t a = 0; a < na; a++) s += cfv[a * n + h];
          out[h] = s * mean;
        }
    }
    for (size_t a = 0; a < na; a++)
      for (size_t h = 0; h < n; h++) {
        float x = r[a * n + h];
        float disc = x > 0.0f ? d.pos : d.neg;
        r[a * n + h] = x * disc + cfv[a * n + h] - out[h];
      }
    });
  }
}

// cfr.rs:290-301.
static void own_node(const Ctx& ctx, const Node& node, int p, const float* opp_reach, size_t nq, const Mode& mode,
                     float* out, size_t n) {
  size_t na = node.num_children;
  Buf cfv(na * n);
  for (size_t a = 0; a < na; a++) traverse(ctx, node.first_child + a, p, opp_reach, nq, mode, cfv.data() + a * n, n);
  if (n == 0) return;
  own_node_update(ctx, node, n, cfv.data(), mode, out);
}

// cfr.rs:384-433.
static void opponent_node(const Ctx& ctx, const Node& node, int p, const float* opp_reach, size_t nq,
                          const Mode& mode, float* out, size_t n) {
  size_t na = node.num_children;
  Buf s(na * nq);
  if (nq > 0) {
    if (mode.kind == MODE_CFR) {
      load_current_strategy(*ctx.store, node, nq, s.data());
      const Discount& d = mode.d;
      update_strat(*ctx.store, node, nq, [&](float* ss) {
        for (size_t a = 0; a < na; a++)
          for (size_t h = 0; h < nq; h++) {
            float& x = ss[a * nq + h];
            if (d.reach_weighted)
              x = x * d.strat + s[a * nq + h] * opp_reach[h];
            else
              x = x * d.strat + s[a * nq + h];
          }
      });
    } else {
      load_strat(*ctx.store, node, nq, s.data());
      normalize_in_place(s.data(), na, nq);
    }
    for (size_t a = 0; a < na; a++)
      for (size_t h = 0; h < nq; h++) s[a * nq + h] *= opp_reach[h];
  }
  for (size_t h = 0; h < n; h++) out[h] = 0.0f;
  Buf tmp(n);
  for (size_t a = 0; a < na; a++) {
    const float* r_a = s.data() + a * nq;
    bool all_zero = true;
    for (size_t h = 0; h < nq; h++)
      if (r_a[h] != 0.0f) {
        all_zero = false;
        break;
      }
    if (all_zero) continue;
    traverse(ctx, node.first_child + a, p, r_a, nq, mode, tmp.data(), n);
    for (size_t h = 0; h < n; h++) out[h] += tmp[h];
  }
}

// cfr.rs:435-479.
static void chance(const Ctx& ctx, const Node& node, int p, const float* opp_reach, size_t nq, const Mode& mode,
                   float* out, size_t n) {
  bool all_zero = true;
  for (size_t h = 0; h < nq; h++)
    if (opp_reach[h] != 0.0f) {
      all_zero = false;
      break;
    }
  if (n == 0 || all_zero) {
    for (size_t h = 0; h < n; h++) out[h] = 0.0f;
    return;
  }
  int o = p ^ 1;
  float factor = node.chance_factor;
  size_t k = node.num_children;
  std::vector<float> rows(k * n);
  auto child_task = [&](size_t i) {
    size_t c = node.first_child + i;
    int card = ctx.tree->nodes[c].edge_card;
    Buf r(opp_reach, nq);
    for (size_t h = 0; h < nq; h++) r[h] *= factor;
    for (uint32_t h : ctx.hands->blocked[o][card]) r[h] = 0.0f;
    float* row = rows.data() + i * n;
    traverse(ctx, c, p, r.data(), nq, mode, row, n);
    for (uint32_t h : ctx.hands->blocked[p][card]) row[h] = 0.0f;
  };
  if (omp_in_parallel()) {
#pragma omp taskloop grainsize(1)
    for (size_t i = 0; i < k; i++) child_task(i);
  } else {
    for (size_t i = 0; i < k; i++) child_task(i);
  }
  std::vector<double> acc(n, 0.0);
  for (size_t i = 0; i < k; i++)
    for (size_t h = 0; h < n; h++) acc[h] += (double)rows[i * n + h];
  for (auto& pr : ctx.tree->chance[node.slot].iso) {
    const float* row = rows.data() + (size_t)pr.first * n;
    const std::vector<uint16_t>& perm = ctx.iso->perm[p][pr.second];
    for (size_t h = 0; h < n; h++) acc[h] += (double)row[perm[h]];
  }
  for (size_t h = 0; h < n; h++) out[h] = (float)acc[h];
}

// river.rs: breadth-first river subtree.
struct RItem {
  uint32_t id, first_child, reach;
  bool dead;
};
struct RScratch {
  std::vector<RItem> items;
  std::vector<float> reach, vals, strat;
  struct Group {
    uint32_t reach, sd, fd;
  };
  std::vector<Group> groups;
  std::vector<uint32_t> group_of;
};

static void set_len_unzeroed(std::vector<float>& v, size_t len) { v.resize(len); }

static void river_run(const Ctx& ctx, size_t root, int p, const float* opp_reach, size_t nq, const Mode& mode,
                      float* out, size_t n) {
  static thread_local RScratch S;
  const auto& nodes = ctx.tree->nodes;
  auto& items = S.items;
  auto& reach = S.reach;
  auto& vals = S.vals;
  auto& strat = S.strat;
  auto& groups = S.groups;
  auto& group_of = S.group_of;
  // Phase 0 (river.rs:72-90).
  items.clear();
  bool root_dead = true;
  for (size_t h = 0; h < nq; h++)
    if (opp_reach[h] != 0.0f) {
      root_dead = false;
      break;
    }
  items.push_back(RItem{(uint32_t)root, 0, 0, root_dead});
  size_t reach_slots = 1;
  for (size_t k = 0; k < items.size(); k++) {
    const Node& node = nodes[items[k].id];
    if (node.kind == K_PLAYER) {
      items[k].first_child = (uint32_t)items.size();
      for (uint32_t c = node.first_child; c < node.first_child + node.num_children; c++)
        items.push_back(RItem{c, 0, 0, false});
      if (node.player != p) reach_slots += node.num_children;
    }
  }
  // Phase 1 (river.rs:92-161).
  set_len_unzeroed(reach, reach_slots * nq);
  std::memcpy(reach.data(), opp_reach, nq * sizeof(float));
  size_t next_slot = 1;
  for (size_t k = 0; k < items.size(); k++) {
    RItem it = items[k];
    const Node& node = nodes[it.id];
    if (node.kind != K_PLAYER) continue;
    size_t na = node.num_children;
    size_t fc = it.first_child;
    if (it.dead) {
      for (size_t c = fc; c < fc + na; c++) items[c].dead = true;
      continue;
    }
    if (node.player == p) {
      for (size_t c = fc; c < fc + na; c++) items[c].reach = it.reach;
      continue;
    }
    set_len_unzeroed(strat, na * nq);
    if (mode.kind == MODE_CFR) {
      load_current_strategy(*ctx.store, node, nq, strat.data());
      const float* r = reach.data() + (size_t)it.reach * nq;
      float g = mode.d.strat;
      update_strat(*ctx.store, node, nq, [&](float* ss) {
        for (size_t a = 0; a < na; a++)
          for (size_t h = 0; h < nq; h++) {
            float& x = ss[a * nq + h];
            if (mode.d.reach_weighted)
              x = x * g + strat[a * nq + h] * r[h];
            else
              x = x * g + strat[a * nq + h];
          }
      });
    } else {
      load_strat(*ctx.store, node, nq, strat.data());
      normalize_in_place(strat.data(), na, nq);
    }
    size_t parent = (size_t)it.reach * nq;
    for (size_t a = 0; a < na; a++) {
      size_t slot = next_slot++;
      float* dst = reach.data() + slot * nq;
      const float* src = reach.data() + parent;
      const float* row = strat.data() + a * nq;
      bool any = false;
      for (size_t h = 0; h < nq; h++) {
        dst[h] = src[h] * row[h];
        any |= dst[h] != 0.0f;
      }
      items[fc + a].reach = (uint32_t)slot;
      items[fc + a].dead = !any;
    }
  }
  // Phase 2 (river.rs:163-249).
  vals.assign(items.size() * n, 0.0f);
  if (n == 0) return;
  auto reach_of = [&](uint32_t slot) { return reach.data() + (size_t)slot * nq; };
  group_of.assign(reach_slots, NONE);
  groups.clear();
  int64_t board_table = -1;
  for (size_t k = 0; k < items.size(); k++) {
    const RItem& it = items[k];
    if (it.dead) continue;
    const Node& node = nodes[it.id];
    bool is_showdown;
    if (node.kind == K_SHOWDOWN)
      is_showdown = true;
    else if (node.kind == K_FOLD)
      is_showdown = false;
    else
      continue;
    if (is_showdown) board_table = (int64_t)node.offset;
    uint32_t g = group_of[it.reach];
    bool fits = g != NONE && (is_showdown ? groups[g].sd == NONE : groups[g].fd == NONE);
    size_t gi;
    if (fits) {
      gi = g;
    } else {
      group_of[it.reach] = (uint32_t)groups.size();
      groups.push_back(RScratch::Group{it.reach, NONE, NONE});
      gi = groups.size() - 1;
    }
    if (is_showdown)
      groups[gi].sd = (uint32_t)k;
    else
      groups[gi].fd = (uint32_t)k;
  }
  // Groups with a showdown first (the order inside each class does not
  // change any value: lanes are independent).
  std::stable_partition(groups.begin(), groups.end(), [](const RScratch::Group& g) { return g.sd != NONE; });
  size_t split = 0;
  while (split < groups.size() && groups[split].sd != NONE) split++;
  if (board_table >= 0) {
    const StrengthTable& table = (*ctx.tables)[board_table];
    for (size_t c0 = 0; c0 < split; c0 += LANES) {
      size_t c1 = std::min(split, c0 + LANES);
      std::vector<const float*> reaches;
      std::vector<double> win, lose, tie;
      std::vector<float*> outs;
      std::vector<std::pair<double, float*>> folds;
      std::vector<bool> has_fold;
      for (size_t g = c0; g < c1; g++) {
        reaches.push_back(reach_of(groups[g].reach));
        double w, l, t;
        showdown_payoffs(ctx, nodes[items[groups[g].sd].id], p, w, l, t);
        win.push_back(w);
        lose.push_back(l);
        tie.push_back(t);
        outs.push_back(vals.data() + (size_t)groups[g].sd * n);
        if (groups[g].fd != NONE) {
          folds.push_back({fold_payoff(ctx, nodes[items[groups[g].fd].id], p), vals.data() + (size_t)groups[g].fd * n});
          has_fold.push_back(true);
        } else {
          folds.push_back({0.0, nullptr});
          has_fold.push_back(false);
        }
      }
      showdown_batch(*ctx.hands, table, p, reaches, win, lose, tie, outs, folds, has_fold);
    }
  }
  for (size_t c0 = split; c0 < groups.size(); c0 += LANES) {
    size_t c1 = std::min(groups.size(), c0 + LANES);
    std::vector<const float*> reaches;
    std::vector<double> payoffs;
    std::vector<float*> outs;
    for (size_t g = c0; g < c1; g++) {
      reaches.push_back(reach_of(groups[g].reach));
      payoffs.push_back(fold_payoff(ctx, nodes[items[groups[g].fd].id], p));
      outs.push_back(vals.data() + (size_t)groups[g].fd * n);
    }
    fold_batch(*ctx.hands, p, reaches, payoffs, outs);
  }
  // Phase 3 (river.rs:251-275).
  for (size_t k = items.size(); k-- > 0;) {
    RItem it = items[k];
    const Node& node = nodes[it.id];
    if (node.kind != K_PLAYER || it.dead) continue;
    size_t na = node.num_children;
    size_t fc = it.first_child;
    float* me = vals.data() + k * n;
    const float* child = vals.data() + fc * n;
    if (node.player != p) {
      for (size_t h = 0; h < n; h++) me[h] = 0.0f;
      for (size_t a = 0; a < na; a++)
        for (size_t h = 0; h < n; h++) me[h] += child[a * n + h];
      continue;
    }
    own_node_update(ctx, node, n, child, mode, me);
  }
  std::memcpy(out, vals.data(), n * sizeof(float));
}

// cfr.rs:259-288.
static void traverse(const Ctx& ctx, size_t id, int p, const float* opp_reach, size_t nq, const Mode& mode, float* out,
                     size_t n) {
  const Node& node = ctx.tree->nodes[id];
  if (node.kind == K_PLAYER) {
    bool all_zero = true;
    for (size_t h = 0; h < nq; h++)
      if (opp_reach[h] != 0.0f) {
        all_zero = false;
        break;
      }
    if (all_zero) {
      for (size_t h = 0; h < n; h++) out[h] = 0.0f;
      return;
    }
  }
  switch (node.kind) {
    case K_FOLD: eval_fold(*ctx.hands, p, opp_reach, fold_payoff(ctx, node, p), out); break;
    case K_SHOWDOWN: {
      double w, l, t;
      showdown_payoffs(ctx, node, p, w, l, t);
      eval_showdown(*ctx.hands, (*ctx.tables)[node.offset], p, opp_reach, w, l, t, out);
      break;
    }
    case K_CHANCE: chance(ctx, node, p, opp_reach, nq, mode, out, n); break;
    case K_PLAYER:
      if (ctx.batch_river && node.street == RIVER)
        river_run(ctx, id, p, opp_reach, nq, mode, out, n);
      else if (node.player == p)
        own_node(ctx, node, p, opp_reach, nq, mode, out, n);
      else
        opponent_node(ctx, node, p, opp_reach, nq, mode, out, n);
      break;
  }
}

// ---------------------------------------------------------------- solver
uint32_t next_check_gap(bool has_prev, uint32_t t0, double e0, uint32_t t, double e, double target, uint32_t max_gap) {
  uint32_t min_gap = std::max(max_gap / 4, 1u);
  if (!has_prev) return max_gap;
  if (!(e < e0 && e > target && t > t0 && target > 0.0)) return max_gap;
  double k = std::log(e0 / e) / std::log((double)t / (double)t0);
  double predicted = (double)t * std::pow(e / target, 1.0 / k);
  double gap = std::ceil(predicted - (double)t);
  if (std::isfinite(gap)) {
    double g = gap > 0.0 ? gap : 0.0;
    // Rust `as u32` saturates.
    uint32_t gu = g >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)g;
    return std::min(std::max(gu, min_gap), max_gap);
  }
  return max_gap;
}

static bool validate(const SolveConfig& cfg, HandSet& hands, int& err, std::string& msg) {
  size_t n = cfg.board.size();
  if (n < 3 || n > 5) {
    err = ERR_INVALID_BOARD;
    msg = "invalid board: " + std::to_string(n) + " cards";
    return false;
  }
  uint64_t set = 0;
  for (int c : cfg.board) {
    if (c < 0 || c >= 52) {
      err = ERR_INVALID_BOARD;
      msg = "invalid board: bad card";
      return false;
    }
    set |= 1ull << c;
  }
  if ((size_t)__builtin_popcountll(set) != n) {
    err = ERR_INVALID_BOARD;
    msg = "invalid board: duplicate cards";
    return false;
  }
  if (street_from_board_len((int)n) != cfg.root.street) {
    err = ERR_INVALID_BOARD;
    msg = "invalid board: board doesn't match the root street";
    return false;
  }
  hands.build(cfg.ranges, set, cfg.prune, cfg.keep);
  for (int p = 0; p < 2; p++)
    if (hands.len(p) == 0) {
      err = ERR_EMPTY_RANGE;
      msg = "player " + std::to_string(p) + " has an empty range";
      return false;
    }
  if (hands.num_combinations <= 0.0) {
    err = ERR_EMPTY_RANGE;
    msg = "player 0 has an empty range";
    return false;
  }
  return true;
}

static TreeParams make_params(const SolveConfig& cfg, const HandSet& hands, const Isomorphism& iso) {
  TreeParams tp;
  tp.root_street = cfg.root.street;
  tp.root_board = &cfg.board;
  tp.menu = &cfg.menu;
  tp.future_menu = cfg.has_future_menu ? &cfg.future_menu : &cfg.menu;
  tp.big_blind = cfg.big_blind;
  tp.num_hands[0] = hands.len(0);
  tp.num_hands[1] = hands.len(1);
  tp.rake_rate = cfg.rake_rate;
  tp.rake_cap = cfg.rake_cap;
  tp.iso = &iso;
  tp.sampled = cfg.sampled;
  tp.sample_turn = cfg.sample_turn;
  tp.sample_river = cfg.sample_river;
  return tp;
}

static bool compressed_mode(const SolveConfig& cfg, const TreeStats& stats) {
  if (cfg.storage == STORAGE_F32) return false;
  if (cfg.storage == STORAGE_COMPRESSED) return true;
  return stats.memory_bytes_f32() > (1ull << 30);
}

bool Solver::estimate(const SolveConfig& cfg, TreeStats& out, int& err, std::string& msg) {
  HandSet hands;
  if (!validate(cfg, hands, err, msg)) return false;
  Isomorphism iso;
  iso.build(hands, cfg.isomorphism);
  TreeParams tp = make_params(cfg, hands, iso);
  TreeStats st;
  std::vector<int> dealt;
  ChaChaRng count_rng(0);  // count_tree's own generator (tree.rs:338-343)
  tp.rng = &count_rng;
  count_player(tp, cfg.root, dealt, st);
  st.compressed = compressed_mode(cfg, st);
  out = st;
  return true;
}

std::unique_ptr<Solver> Solver::create(const SolveConfig& cfg, int& err, std::string& msg) {
  auto s = std::make_unique<Solver>();
  s->config = cfg;
  if (!validate(s->config, s->hands, err, msg)) return nullptr;
  s->iso.build(s->hands, s->config.isomorphism);
  TreeParams tp = make_params(s->config, s->hands, s->iso);
  TreeStats st;
  std::vector<int> dealt;
  ChaChaRng count_rng(0);  // count_tree's own generator (tree.rs:338-343)
  tp.rng = &count_rng;
  count_player(tp, s->config.root, dealt, st);
  st.compressed = compressed_mode(s->config, st);
  uint64_t needed = st.memory_bytes();
  if (needed > s->config.max_memory_bytes) {
    err = ERR_TOO_LARGE;
    char buf[160];
    snprintf(buf, sizeof buf, "game tree needs ~%.2f GB but the limit is %.2f GB", (double)needed / 1e9,
             (double)s->config.max_memory_bytes / 1e9);
    msg = buf;
    return nullptr;
  }
  ChaChaRng build_rng(s->config.sampled ? s->config.sample_seed : 0);  // Builder::new (tree.rs:415-420)
  tp.rng = &build_rng;
  Builder b(tp);
  b.build(s->config.root);
  s->tree = std::move(b.tree);
  s->stats = st;
  s->store.compressed = st.compressed;
  if (st.compressed) {
    s->store.rq.assign(s->tree.storage_len, 0);
    s->store.sq.assign(s->tree.storage_len, 0);
    s->store.rscale.assign(s->tree.num_player_nodes, 0.0f);
    s->store.sscale.assign(s->tree.num_player_nodes, 0.0f);
  } else {
    s->store.regrets.assign(s->tree.storage_len, 0.0f);
    s->store.strat.assign(s->tree.storage_len, 0.0f);
  }
  s->tables.resize(s->tree.boards.size());
  for (size_t i = 0; i < s->tree.boards.size(); i++) s->tables[i].build(s->hands, s->tree.boards[i]);
  s->iterations = 0;
  s->last_exploitability = INFINITY;
  err = ERR_NONE;
  return s;
}

void Solver::traverse_root(int p, int mode, uint32_t t, float* out) {
  Ctx ctx{&tree, &store, &hands, &tables, &iso, (double)config.root.pot / 2.0, 1.0 / hands.num_combinations,
          batch_river};
  Mode m{(ModeKind)mode, Discount::make(t, config.dcfr)};
  par_region([&] { traverse(ctx, 0, p, hands.weights[p ^ 1].data(), hands.len(p ^ 1), m, out, hands.len(p)); });
}

// cpu_iteration (lib.rs:577-585).
void Solver::iterate(uint32_t n) {
  for (uint32_t i = 0; i < n; i++) {
    iterations += 1;
    Discount d = Discount::make(iterations, config.dcfr);
    Ctx ctx{&tree, &store, &hands, &tables, &iso, (double)config.root.pot / 2.0, 1.0 / hands.num_combinations,
            batch_river};
    Mode m{MODE_CFR, d};
    for (int p = 0; p < 2; p++) {
      std::vector<float> out(hands.len(p));
      par_region(
          [&] { traverse(ctx, 0, p, hands.weights[p ^ 1].data(), hands.len(p ^ 1), m, out.data(), hands.len(p)); });
    }
  }
}

// cfr.rs:482-502.
static void root_values_mode(const Solver& s, ModeKind mk, double res[2]) {
  Ctx ctx{&s.tree, const_cast<Storage*>(&s.store), &s.hands, &s.tables, &s.iso, (double)s.config.root.pot / 2.0,
          1.0 / s.hands.num_combinations, s.batch_river};
  Mode m{mk, Discount{0, 0, 0, false}};
  for (int p = 0; p < 2; p++) {
    std::vector<float> v(s.hands.len(p));
    par_region(
        [&] { traverse(ctx, 0, p, s.hands.weights[p ^ 1].data(), s.hands.len(p ^ 1), m, v.data(), s.hands.len(p)); });
    double acc = -0.0;
    for (size_t h = 0; h < v.size(); h++) acc += (double)v[h] * (double)s.hands.weights[p][h];
    res[p] = acc;
  }
}

double Solver::exploitability() const {
  double br[2];
  root_values_mode(*this, MODE_BR, br);
  if (raked()) {
    double ev[2];
    root_values_mode(*this, MODE_AVG, ev);
    return ((br[0] - ev[0]) + (br[1] - ev[1])) / 2.0;
  }
  return (br[0] + br[1]) / 2.0;
}

void Solver::root_values(double out[2]) const { root_values_mode(*this, MODE_AVG, out); }

// run_solve (lib.rs:594-642).
Progress Solver::solve(uint32_t max_iterations, double target_pct, uint32_t check_every0,
                       const std::function<bool(const Progress&)>* on_progress) {
  double pot = (double)config.root.pot;
  uint32_t check_every = std::max(check_every0, 1u);
  Progress progress{iterations, max_iterations, last_exploitability, 100.0 * last_exploitability / pot, false};
  double target = target_pct * pot / 100.0;
  uint32_t next_check = iterations + check_every;
  bool has_last = false;
  uint32_t last_t = 0;
  double last_e = 0.0;
  while (iterations < max_iterations) {
    iterate(1);
    bool last = iterations >= max_iterations;
    if (iterations >= next_check || last) {
      double e = exploitability();
      last_exploitability = e;
      progress.iteration = iterations;
      progress.exploitability = e;
      progress.exploitability_pct = 100.0 * e / pot;
      bool done = progress.exploitability_pct <= target_pct || last;
      progress.finished = done;
      bool keep_going = on_progress ? (*on_progress)(progress) : true;
      if (done || !keep_going) {
        progress.finished = true;
        return progress;
      }
      uint32_t t = iterations;
      next_check = t + next_check_gap(has_last, last_t, last_e, t, e, target, check_every);
      has_last = true;
      last_t = t;
      last_e = e;
    }
  }
  progress.finished = true;
  return progress;
}

// lib.rs:735-743.
std::vector<float> Solver::average_strategy(size_t id, size_t n) const {
  const Node& node = tree.nodes[id];
  std::vector<float> s(node.num_children * n, 0.0f);
  if (n > 0) {
    load_strat(store, node, n, s.data());
    normalize_in_place(s.data(), node.num_children, n);
  }
  return s;
}

// lib.rs:746-825.
bool Solver::walk(const std::vector<Step>& path, size_t& id_out, std::vector<float> reach[2],
                  std::vector<uint32_t> to_canon[2], std::string& err) const {
  size_t id = 0;
  reach[0] = hands.weights[0];
  reach[1] = hands.weights[1];
  for (int x = 0; x < 2; x++) {
    to_canon[x].resize(hands.len(x));
    for (size_t i = 0; i < hands.len(x); i++) to_canon[x][i] = (uint32_t)i;
  }
  int suit_map[4] = {0, 1, 2, 3};
  for (size_t depth = 0; depth < path.size(); depth++) {
    const Step& step = path[depth];
    const Node node = tree.nodes[id];
    if (node.kind == K_PLAYER && step.kind == 0) {
      auto actions = tree.actions(id);
      size_t ai = std::find(actions.begin(), actions.end(), step.action) - actions.begin();
      if (ai == actions.size()) {
        err = "bad path: action not available at depth " + std::to_string(depth);
        return false;
      }
      int q = node.player;
      size_t n = hands.len(q);
      auto s = average_strategy(id, n);
      for (size_t i = 0; i < n; i++) reach[q][i] *= s[ai * n + i];
      id = node.first_child + ai;
    } else if (node.kind == K_CHANCE && step.kind == 1) {
      int c = step.card;
      int cc = make_card(card_rank(c), suit_map[card_suit(c)]);
      int canonical = -1;
      for (uint32_t ch = node.first_child; ch < node.first_child + node.num_children; ch++)
        if (tree.nodes[ch].edge_card == cc) {
          id = ch;
          canonical = cc;
          break;
        }
      if (canonical < 0) {
        const ChanceInfo& info = tree.chance[node.slot];
        size_t j = std::find(info.iso_cards.begin(), info.iso_cards.end(), cc) - info.iso_cards.begin();
        if (j == info.iso_cards.size()) {
          err = "bad path: card " + card_to_string(c) + " not in the tree at depth " + std::to_string(depth);
          return false;
        }
        int ci = info.iso[j].first, pair = info.iso[j].second;
        int a = ISO_PAIRS[pair][0], b = ISO_PAIRS[pair][1];
        for (int& s : suit_map) s = s == a ? b : s == b ? a : s;
        for (int x = 0; x < 2; x++) {
          const auto& perm = iso.perm[x][pair];
          std::vector<float> r2(reach[x].size(), 0.0f);
          for (size_t h = 0; h < reach[x].size(); h++) r2[perm[h]] = reach[x][h];
          reach[x] = r2;
          for (auto& t : to_canon[x]) t = perm[t];
        }
        id = node.first_child + ci;
        canonical = tree.nodes[id].edge_card;
      }
      for (int x = 0; x < 2; x++)
        for (uint32_t k : hands.blocked[x][canonical]) reach[x][k] = 0.0f;
    } else {
      err = "bad path: step doesn't match node kind at depth " + std::to_string(depth);
      return false;
    }
  }
  id_out = id;
  return true;
}

bool Solver::is_decision(const std::vector<Step>& path) const {
  size_t id;
  std::vector<float> reach[2];
  std::vector<uint32_t> tc[2];
  std::string err;
  return walk(path, id, reach, tc, err) && tree.nodes[id].kind == K_PLAYER;
}

bool Solver::actions_at(const std::vector<Step>& path, std::vector<Action>& out, std::string& err) const {
  size_t id;
  std::vector<float> reach[2];
  std::vector<uint32_t> tc[2];
  if (!walk(path, id, reach, tc, err)) return false;
  out.clear();
  if (tree.nodes[id].kind == K_PLAYER) out = tree.actions(id);
  return true;
}

// lib.rs:842-899.
bool Solver::query(const std::vector<Step>& path, NodeInfo& info, std::string& err) const {
  size_t id;
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  if (!walk(path, id, reach, to_canon, err)) return false;
  const Node node = tree.nodes[id];
  if (node.kind != K_PLAYER) {
    err = "bad path: not a decision node";
    return false;
  }
  int q = node.player, o = q ^ 1;
  size_t n = hands.len(q);
  size_t na = node.num_children;
  Ctx ctx{&tree, const_cast<Storage*>(&store), &hands, &tables, &iso, (double)config.root.pot / 2.0,
          1.0 / hands.num_combinations, batch_river};
  auto compat = hands.compatible_reach(q, reach[o].data());
  std::vector<std::vector<float>> child_vals(na, std::vector<float>(n, 0.0f));
  Mode m{MODE_AVG, Discount{0, 0, 0, false}};
  for (size_t a = 0; a < na; a++)
    par_region([&] {
      traverse(ctx, node.first_child + a, q, reach[o].data(), hands.len(o), m, child_vals[a].data(), n);
    });
  double offset = ctx.half_pot + (double)node.invest[q];
  auto strat_c = average_strategy(id, n);
  info.ev.assign(na * n, 0.0f);
  info.strategy.assign(na * n, 0.0f);
  info.reach.assign(n, 0.0f);
  for (size_t h = 0; h < n; h++) {
    size_t hc = to_canon[q][h];
    info.reach[h] = reach[q][hc];
    double denom = compat[hc] * ctx.norm;
    for (size_t a = 0; a < na; a++) {
      info.strategy[a * n + h] = strat_c[a * n + hc];
      info.ev[a * n + h] = denom > 0.0 ? (float)((double)child_vals[a][hc] / denom + offset) : 0.0f;
    }
  }
  for (int p = 0; p < 2; p++) {
    double root = -0.0, now = -0.0;
    for (float x : hands.weights[p]) root += (double)x;
    for (float x : reach[p]) now += (double)x;
    info.reach_fraction[p] = root > 0.0 ? now / root : 0.0;
  }
  info.player = q;
  info.actions = tree.actions(id);
  info.combos = hands.combos[q];
  info.pot = config.root.pot + (Chips)node.invest[0] + (Chips)node.invest[1];
  info.invest[0] = node.invest[0];
  info.invest[1] = node.invest[1];
  return true;
}

// lib.rs:903-912.
bool Solver::ranges_after(const std::vector<Step>& path, std::vector<float> out[2], std::string& err) const {
  size_t id;
  std::vector<float> reach[2];
  std::vector<uint32_t> to_canon[2];
  if (!walk(path, id, reach, to_canon, err)) return false;
  for (int p = 0; p < 2; p++) {
    out[p].assign(1326, 0.0f);
    for (size_t h = 0; h < hands.len(p); h++) out[p][hands.combos[p][h]] = reach[p][to_canon[p][h]];
  }
  return true;
}

}  // namespace oracle
