// TEST INFRASTRUCTURE — CPU oracle. Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg may load this code; the product (libdcfr) never
// links it.
//
// Restatement of the reference's poker primitives (AhanDatta/Poker-Trainer,
// crates/holdem): cards (card.rs:46-75), combos and hand classes
// (combo.rs:14-207), the 7-card evaluator (eval.rs:72-198), the postflop bet
// menu (menu.rs:86-133, 193-308, 355-392) and the range notation
// (range.rs:21-264). Every function follows the cited Rust operation for
// operation; compile with -ffp-contract=off (Rust never contracts to FMA).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace oracle {

using Chips = int64_t;

enum Street { PREFLOP = 0, FLOP = 1, TURN = 2, RIVER = 3 };

// Street::board_len / from_board_len (crates/holdem/src/game.rs:37-56).
int street_board_len(Street s);
Street street_from_board_len(int n);

// Card = rank*4 + suit (crates/holdem/src/card.rs:46-48).
inline int card_rank(int c) { return c >> 2; }
inline int card_suit(int c) { return c & 3; }
inline int make_card(int rank, int suit) { return rank * 4 + suit; }
int parse_card(const std::string& s);                    // -1 on error (card.rs:108-121)
bool parse_cards(const std::string& s, std::vector<int>& out);  // card.rs:124-132
std::string card_to_string(int c);

// combo.rs:14-17 and the COMBOS table (combo.rs:19-35): entry = (higher
// card id, lower card id).
inline int combo_index(int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  return hi * (hi - 1) / 2 + lo;
}
struct ComboCards { uint8_t hi, lo; };
const ComboCards* combos_table();  // 1326 entries

// HandClass (combo.rs:58-150) and COMBO_CLASS (combo.rs:186-207).
struct HandClass {
  int hi, lo;
  bool suited;
  static HandClass make(int r1, int r2, bool suited);
  bool is_pair() const { return hi == lo; }
  int grid_index() const;
  static HandClass from_grid_index(int index);
  int num_combos() const;
  std::vector<int> combos() const;
};
const uint8_t* combo_class_table();  // 1326 entries

// Evaluator (crates/holdem/src/eval.rs:72-198): EvalMask lane layout and
// evaluate_mask -> category<<26 | payload.
inline uint64_t eval_card_bit(int c) { return 1ull << (card_suit(c) * 16 + card_rank(c)); }
uint32_t evaluate_mask(uint64_t mask);
uint32_t evaluate_cards(const int* cards, int n);

// Actions (crates/holdem/src/game.rs:76-82).
enum ActionKind { FOLD = 0, CHECK = 1, CALL = 2, RAISE = 3 };
struct Action {
  int kind;
  Chips amount;
  bool operator==(const Action& o) const { return kind == o.kind && amount == o.amount; }
};

// BetSize / StreetSizes / PostflopMenu (crates/holdem/src/menu.rs:16-133).
enum SizeKind { SIZE_POT = 0, SIZE_MULT = 1, SIZE_ALLIN = 2 };
struct BetSize { int kind; double value; };
bool parse_bet_size(const std::string& s, BetSize& out);  // menu.rs:26-50
struct StreetSizes { std::vector<BetSize> bet, raise; };
struct PostflopMenu {
  StreetSizes flop, turn, river;
  uint32_t max_raises = 3;
  double add_allin_threshold = 1.5;
  double force_allin_threshold = 0.15;
  double merge_threshold = 0.1;
  static PostflopMenu defaults();  // menu.rs:119-133
  const StreetSizes& street(Street s) const;
};

// Situation (crates/holdem/src/menu.rs:193-216).
struct Situation {
  Street street;
  Chips pot, to_call, current_bet, max_to, min_raise_to;
  uint32_t num_raises;
  Chips big_blind;
  bool can_raise() const { return max_to > current_bet; }
};

// postflop_actions / postflop_categorized (menu.rs:229-308) with
// finalize_tagged (menu.rs:355-392).
std::vector<Action> postflop_actions(const Situation& sit, const PostflopMenu& menu);

// Range notation (crates/holdem/src/range.rs:201-264): 1326 weights.
bool parse_range(const std::string& s, std::vector<float>& out, std::string* err = nullptr);

}  // namespace oracle
