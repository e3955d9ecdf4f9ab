// TEST INFRASTRUCTURE — CPU oracle. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load this code; the product (libdcfr) never
// links it.
//
// Restatement of the reference's heads-up DCFR solver (AhanDatta/
// Poker-Trainer, crates/solver/src): tree.rs (betting state, arena builder,
// count_tree), hands.rs (hand sets, strength tables), iso.rs (suit
// isomorphism), storage.rs (F32 storage), cfr.rs (discounts, regret
// matching, traversal, chance, exploitability), river.rs (breadth-first
// river subtrees), eval.rs (fold/showdown evaluators) and lib.rs (validate,
// estimate, new, run_solve, walk/query/ranges_after). Chance children are
// traversed in parallel with OpenMP tasks where the reference uses rayon
// (cfr.rs:448); every reduction keeps the reference's order, so results do
// not depend on the thread count.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "holdem.hpp"

namespace oracle {

constexpr uint32_t NONE = 0xFFFFFFFFu;

// DcfrParams (cfr.rs:48-81); defaults = DcfrParams::default.
struct DcfrParams {
  double alpha = 1.5;
  bool beta_clip = false;  // beta = None
  double beta = 0.0;
  double gamma = 3.0;
  bool restart_average = true;
  bool unweighted_average = true;
};

// Discount (cfr.rs:36-107).
struct Discount {
  float pos, neg, strat;
  bool reach_weighted;
  static Discount make(uint32_t t, const DcfrParams& p);
};

// BettingState (tree.rs:17-126).
enum TransitionKind { T_CONTINUE, T_FOLD, T_STREET_OVER };
struct BettingState {
  Street street;
  Chips pot;
  Chips commit[2];
  Chips stack[2];
  Chips current_bet;
  Chips last_raise_inc;
  uint32_t num_raises;
  int to_act;
  bool needs[2];
  static BettingState street_start(Street s, Chips pot, Chips s0, Chips s1, Chips big_blind);
  Situation situation(Chips big_blind) const;
  // apply (tree.rs:93-125): returns the transition, the next state and the
  // chips put in; for T_FOLD `folder` is the player who folded.
  TransitionKind apply(const Action& a, BettingState& next, Chips& put, int& folder) const;
};

enum StorageModeE { STORAGE_F32 = 0, STORAGE_COMPRESSED = 1, STORAGE_AUTO = 2 };

// SolveConfig (lib.rs:74-135).
struct SolveConfig {
  std::vector<int> board;
  std::vector<float> ranges[2];
  BettingState root;
  PostflopMenu menu;
  bool has_future_menu = false;
  PostflopMenu future_menu;
  Chips big_blind = 100;
  float prune = 0.0f;
  std::vector<int> keep[2];
  uint64_t max_memory_bytes = 8ull << 30;
  double rake_rate = 0.0;
  double rake_cap = 0.0;
  int storage = STORAGE_AUTO;
  bool isomorphism = true;
  DcfrParams dcfr;
  // ChanceMode (tree.rs:128-136): sampled = false is Exact.
  bool sampled = false;
  size_t sample_turn = 0, sample_river = 0;
  uint64_t sample_seed = 0;
};

// rand 0.9.5 StdRng = rand_chacha 0.9.0 ChaCha12Rng behind rand_core 0.9's
// BlockRng (a 64-word buffer of four ChaCha blocks), seeded by
// SeedableRng::seed_from_u64 (PCG32 key expansion). Restated from the
// published ChaCha and PCG32 algorithms; tree.rs:415-420 and
// sampling.rs:9-54 are its call sites.
struct ChaChaRng {
  uint32_t key[8];
  uint64_t block_counter = 0;
  uint32_t results[64];
  size_t index = 64;
  explicit ChaChaRng(uint64_t seed);
  uint64_t next_u64();
  double random_f64();  // StandardUniform for f64: [0, 1), 53 bits
};
// The ChaCha block function with `rounds` rounds (20 for ChaCha20, 12 for
// StdRng): key words 4-11, counter words 12-13, stream words 14-15.
void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds, uint32_t out[16]);
// sampling.rs:9-54.
std::vector<int> sample_cards(const std::vector<int>& available, size_t k, ChaChaRng& rng);

// TreeStats (tree.rs:248-274). Node is 56 bytes in the reference's layout
// (tree.rs:154-171: 8+16+8+4+4+4+4+2+2+1 bytes, padded to 8).
constexpr uint64_t NODE_BYTES = 56;
struct TreeStats {
  uint64_t player_nodes = 0, chance_nodes = 0, terminal_nodes = 0, storage_cells = 0;
  bool compressed = false;
  uint64_t total_nodes() const { return player_nodes + chance_nodes + terminal_nodes; }
  uint64_t memory_bytes() const { return storage_cells * (compressed ? 4 : 8) + total_nodes() * NODE_BYTES; }
  uint64_t memory_bytes_f32() const { return storage_cells * 8 + total_nodes() * NODE_BYTES; }
};

enum Kind : uint8_t { K_PLAYER = 0, K_CHANCE = 1, K_FOLD = 2, K_SHOWDOWN = 3 };
enum EdgeKind : uint8_t { E_ROOT = 0, E_ACTION = 1, E_CARD = 2 };

// Node (tree.rs:154-205).
struct Node {
  Kind kind = K_SHOWDOWN;
  uint8_t player = 0;  // Player(q) / Fold(f)
  Street street = RIVER;
  uint16_t num_children = 0;
  uint32_t first_child = 0;
  int32_t invest[2] = {0, 0};
  uint64_t offset = 0;  // player: storage offset; showdown: table index
  uint32_t slot = 0;    // player: storage slot; chance: chance-info index
  float rake = 0.0f;
  float chance_factor = 1.0f;
  EdgeKind edge_kind = E_ROOT;
  Action edge_action{0, 0};
  int edge_card = -1;
};

// ChanceInfo (tree.rs:207-214).
struct ChanceInfo {
  std::vector<std::pair<uint16_t, uint8_t>> iso;
  std::vector<int> iso_cards;
};

struct Tree {
  std::vector<Node> nodes;
  std::vector<ChanceInfo> chance;
  std::vector<std::vector<int>> boards;
  uint64_t storage_len = 0;
  uint32_t num_player_nodes = 0;
  std::vector<Action> actions(size_t id) const;
};

// HandSet (hands.rs:10-126).
struct HandSet {
  std::vector<uint16_t> combos[2];
  std::vector<std::pair<uint8_t, uint8_t>> cards[2];
  std::vector<float> weights[2];
  std::vector<uint32_t> same[2];
  std::vector<std::vector<uint32_t>> blocked[2];
  std::vector<uint32_t> lookup[2];
  double num_combinations = 0.0;
  void build(const std::vector<float> ranges[2], uint64_t board_set, float prune, const std::vector<int> keep[2]);
  size_t len(int p) const { return combos[p].size(); }
  std::vector<double> compatible_reach(int p, const float* opp_reach) const;
};

// eval::Entry (eval.rs:11-18) and StrengthTable (hands.rs:128-158).
struct Entry {
  uint32_t strength;
  uint16_t idx;
  uint8_t c1, c2;
};
struct StrengthTable {
  std::vector<Entry> lists[2];
  void build(const HandSet& hands, const std::vector<int>& board);
};

// Isomorphism (iso.rs:236-301).
extern const uint8_t ISO_PAIRS[6][2];
int iso_pair_index(int a, int b);
int swap_card(int card, int a, int b);
std::vector<std::pair<int, int>> board_symmetric_pairs(const std::vector<int>& board);
std::vector<int> iso_orbit(const std::vector<int>& board, int combo);
struct IsoRef {
  int card, canonical, pair;
};
struct Isomorphism {
  bool enabled = false;
  bool range_symmetric[6] = {false, false, false, false, false, false};
  std::vector<uint16_t> perm[2][6];
  void build(const HandSet& hands, bool enabled);
  void chance_cards(const std::vector<int>& board, const std::vector<int>& available, std::vector<int>& canonical,
                    std::vector<IsoRef>& refs) const;
};

// Storage (storage.rs:87-98): F32, or Compressed (16-bit values with one
// f32 scale per player node slot: regrets i16 scaled by max|r| / 32767,
// strategy sums u16 scaled by max / 65535).
struct Storage {
  bool compressed = false;
  std::vector<float> regrets, strat;  // F32
  std::vector<int16_t> rq;            // Compressed
  std::vector<uint16_t> sq;
  std::vector<float> rscale, sscale;  // per player node slot
};

enum ModeKind { MODE_CFR = 0, MODE_BR = 1, MODE_AVG = 2 };
struct Mode {
  ModeKind kind;
  Discount d;
};

struct Ctx;

// next_check_gap (lib.rs:158-172).
uint32_t next_check_gap(bool has_prev, uint32_t t0, double e0, uint32_t t, double e, double target, uint32_t max_gap);

// Terminal evaluators (eval.rs), exposed for the evaluator tests.
void eval_fold(const HandSet& hs, int p, const float* opp_reach, double payoff, float* out);
void eval_showdown(const HandSet& hs, const StrengthTable& table, int p, const float* opp_reach, double win,
                   double lose, double tie, float* out);
void fold_batch(const HandSet& hs, int p, const std::vector<const float*>& reaches, const std::vector<double>& payoffs,
                const std::vector<float*>& outs);
void showdown_batch(const HandSet& hs, const StrengthTable& table, int p, const std::vector<const float*>& reaches,
                    const std::vector<double>& win, const std::vector<double>& lose, const std::vector<double>& tie,
                    const std::vector<float*>& outs, const std::vector<std::pair<double, float*>>& folds,
                    const std::vector<bool>& has_fold);

struct Step {
  int kind;  // 0 action, 1 card
  Action action;
  int card;
};

// NodeInfo (lib.rs:220-240).
struct NodeInfo {
  int player;
  std::vector<Action> actions;
  std::vector<uint16_t> combos;
  std::vector<float> strategy, ev, reach;
  double reach_fraction[2];
  Chips pot;
  Chips invest[2];
};

struct Progress {
  uint32_t iteration, max_iterations;
  double exploitability, exploitability_pct;
  bool finished;
};

enum SolverErr { ERR_NONE = 0, ERR_EMPTY_RANGE = 1, ERR_INVALID_BOARD = 2, ERR_TOO_LARGE = 3, ERR_BAD_PATH = 4 };

class Solver {
 public:
  // Solver::new (lib.rs:365-396); on failure returns null and sets err/msg.
  static std::unique_ptr<Solver> create(const SolveConfig& cfg, int& err, std::string& msg);
  static bool estimate(const SolveConfig& cfg, TreeStats& out, int& err, std::string& msg);

  Progress solve(uint32_t max_iterations, double target_pct, uint32_t check_every,
                 const std::function<bool(const Progress&)>* on_progress);
  void iterate(uint32_t n);  // cpu_iteration x n
  double exploitability() const;
  void root_values(double out[2]) const;
  bool query(const std::vector<Step>& path, NodeInfo& out, std::string& err) const;
  bool ranges_after(const std::vector<Step>& path, std::vector<float> out[2], std::string& err) const;
  bool actions_at(const std::vector<Step>& path, std::vector<Action>& out, std::string& err) const;
  bool is_decision(const std::vector<Step>& path) const;
  void traverse_root(int p, int mode, uint32_t t, float* out);

  SolveConfig config;
  HandSet hands;
  Isomorphism iso;
  Tree tree;
  Storage store;
  std::vector<StrengthTable> tables;
  TreeStats stats;
  uint32_t iterations = 0;
  double last_exploitability;
  bool batch_river = true;

 private:
  bool walk(const std::vector<Step>& path, size_t& node, std::vector<float> reach[2], std::vector<uint32_t> to_canon[2],
            std::string& err) const;
  std::vector<float> average_strategy(size_t id, size_t n) const;
  bool raked() const { return config.rake_rate > 0.0 && config.rake_cap > 0.0; }
};

void set_num_threads(int n);
int get_num_threads();

}  // namespace oracle
