// Host-side game model of libdcfr: bet menu, betting state, the game tree
// in the reference's node order, hand sets and suit isomorphism. It is the
// input of the device plan (plan.hpp); nothing here runs per iteration.
//
// Semantics follow AhanDatta/Poker-Trainer: crates/holdem/src/menu.rs:229-392
// (actions), crates/solver/src/tree.rs:49-573 (betting state, count_tree,
// Builder), crates/solver/src/hands.rs:35-125 (HandSet) and
// crates/solver/src/iso.rs:86-141 (Isomorphism). Node order and storage
// offsets equal the reference's so storage can be exchanged in its layout.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/dcfr.h"

namespace dcfr {

// N_LEAF: a depth-limited solve's cut (the deal of leaf_street), valued by
// the leaf-value network instead of a subtree.
enum : uint8_t { N_PLAYER = 0, N_CHANCE = 1, N_FOLD = 2, N_SHOWDOWN = 3, N_LEAF = 4 };
constexpr uint32_t NO = 0xFFFFFFFFu;

struct Act {
  int32_t kind;
  int64_t amount;
  bool operator==(const Act& o) const { return kind == o.kind && amount == o.amount; }
};

struct Betting {
  int street;
  int64_t pot, commit[2], stack[2], current_bet, last_raise_inc;
  uint32_t num_raises;
  int to_act;
  bool needs[2];
};

struct GNode {
  uint8_t kind = N_SHOWDOWN;
  uint8_t player = 0;  // acting player / folder
  uint8_t street = DCFR_RIVER;
  uint16_t nchild = 0;
  uint32_t first = 0;
  int32_t invest[2] = {0, 0};
  uint64_t ref_offset = 0;  // player: storage offset in the reference layout
  uint32_t index = 0;       // player: player-node ordinal; chance: chance ordinal; showdown: board
  float rake = 0.0f;
  float factor = 1.0f;
  int card = -1;  // edge card (children of chance nodes)
  Act act{0, 0};  // edge action
  uint32_t parent = NO;
};

struct ChanceIso {
  std::vector<uint16_t> ci;    // canonical child index
  std::vector<uint8_t> pair;   // suit pair
  std::vector<uint8_t> cards;  // the isomorphic card
};

struct Stats {
  uint64_t player = 0, chance = 0, terminal = 0, cells = 0;
};

struct Game {
  dcfr_config cfg;
  std::vector<int> board;
  // Hands (hands.rs:10-30).
  int n[2] = {0, 0};
  std::vector<uint16_t> combos[2];
  std::vector<uint8_t> c1[2], c2[2];  // higher / lower card id of each hand
  std::vector<float> weights[2];
  std::vector<uint32_t> same[2];
  std::vector<uint32_t> lookup[2];
  std::vector<std::vector<uint32_t>> blocked[2];  // per card, hands holding it (ascending)
  double num_combinations = 0.0;
  double norm = 0.0, half_pot = 0.0;
  // Isomorphism (iso.rs:236-242).
  bool iso_enabled = false;
  bool sym[6] = {false, false, false, false, false, false};
  std::vector<uint16_t> perm[2][6];
  // Tree (tree.rs:216-223).
  std::vector<GNode> nodes;
  std::vector<ChanceIso> chance;
  std::vector<std::vector<int>> boards;
  uint64_t storage_len = 0;
  uint32_t player_nodes = 0;
  Stats stats;
  bool compressed = false;
  // Depth limit: the deal of this street ends the tree in N_LEAF nodes
  // (-1: no limit). Leaves in creation order: node id, pot, effective stack.
  int leaf_street = -1;
  struct Leaf {
    uint32_t node;
    int64_t pot, stack;
  };
  std::vector<Leaf> leaves;

  std::vector<Act> actions(uint32_t id) const;
};

// Builds everything; on failure returns a DCFR_ERR_* code and a message.
int build_game(const dcfr_config& cfg, Game& g, std::string& msg, bool build_tree, int leaf_street = -1);

// Memory estimate of the reference (TreeStats::memory_bytes, tree.rs:264-268).
uint64_t reference_memory_bytes(const Stats& s, bool compressed);

// Postflop action list for a betting state (menu.rs:264-308 via
// tree.rs:298-300).
std::vector<Act> state_actions(const Betting& st, const dcfr_menu& menu, int64_t big_blind);

// Average strategy of a block (cfr.rs:124-154 normalize_in_place), host
// side, for the path walk of queries.
void normalize_rows(float* s, int na, int n);

// Decision nodes in the reference's storage order (Node::offset). build_game
// gives each decision node its ordinal (`index`) and its storage offset at
// the same step, so the ordinal orders them: no sort needed.
std::vector<uint32_t> players_in_storage_order(const Game& g);

}  // namespace dcfr
