// TEST INFRASTRUCTURE — CPU oracle (see holdem.hpp). Restates
// crates/holdem/src/{card,combo,eval,menu,range}.rs of AhanDatta/Poker-Trainer.
#include "holdem.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <utility>

namespace oracle {

static const char RANK_CHARS[] = "23456789TJQKA";
static const char SUIT_CHARS[] = "cdhs";

int street_board_len(Street s) {
  switch (s) {
    case FLOP: return 3;
    case TURN: return 4;
    case RIVER: return 5;
    default: return 0;
  }
}

Street street_from_board_len(int n) {
  switch (n) {
    case 0: return PREFLOP;
    case 3: return FLOP;
    case 4: return TURN;
    default: return RIVER;
  }
}

static int parse_rank(char c) {
  c = (char)std::toupper((unsigned char)c);
  for (int i = 0; i < 13; i++)
    if (RANK_CHARS[i] == c) return i;
  return -1;
}

static int parse_suit(char c) {
  c = (char)std::tolower((unsigned char)c);
  for (int i = 0; i < 4; i++)
    if (SUIT_CHARS[i] == c) return i;
  return -1;
}

// card.rs:108-121 (the string is trimmed first).
int parse_card(const std::string& s0) {
  size_t a = 0, b = s0.size();
  while (a < b && std::isspace((unsigned char)s0[a])) a++;
  while (b > a && std::isspace((unsigned char)s0[b - 1])) b--;
  if (b - a != 2) return -1;
  int r = parse_rank(s0[a]), su = parse_suit(s0[a + 1]);
  if (r < 0 || su < 0) return -1;
  return make_card(r, su);
}

// card.rs:124-132: whitespace and commas dropped, then pairs of chars.
bool parse_cards(const std::string& s, std::vector<int>& out) {
  std::string compact;
  for (char c : s)
    if (!std::isspace((unsigned char)c) && c != ',') compact.push_back(c);
  if (compact.size() % 2 != 0) return false;
  out.clear();
  for (size_t i = 0; i < compact.size(); i += 2) {
    int c = parse_card(compact.substr(i, 2));
    if (c < 0) return false;
    out.push_back(c);
  }
  return true;
}

std::string card_to_string(int c) {
  std::string s;
  s.push_back(RANK_CHARS[card_rank(c)]);
  s.push_back(SUIT_CHARS[card_suit(c)]);
  return s;
}

// COMBOS (combo.rs:19-35).
static ComboCards g_combos[1326];
static uint8_t g_combo_class[1326];
static bool g_tables_ready = [] {
  for (int hi = 1; hi < 52; hi++)
    for (int lo = 0; lo < hi; lo++) g_combos[hi * (hi - 1) / 2 + lo] = ComboCards{(uint8_t)hi, (uint8_t)lo};
  // build_combo_class (combo.rs:186-204).
  for (int i = 0; i < 1326; i++) {
    int a = g_combos[i].hi, b = g_combos[i].lo;
    int hi = card_rank(a), lo = card_rank(b);
    bool suited = card_suit(a) == card_suit(b);
    int r_hi = 12 - hi, r_lo = 12 - lo;
    g_combo_class[i] = (uint8_t)(hi == lo ? r_hi * 13 + r_hi : suited ? r_hi * 13 + r_lo : r_lo * 13 + r_hi);
  }
  return true;
}();

const ComboCards* combos_table() { return g_combos; }
const uint8_t* combo_class_table() { return g_combo_class; }

// HandClass (combo.rs:69-150).
HandClass HandClass::make(int r1, int r2, bool suited) {
  int hi = r1 >= r2 ? r1 : r2, lo = r1 >= r2 ? r2 : r1;
  return HandClass{hi, lo, suited && hi != lo};
}

int HandClass::grid_index() const {
  int r_hi = 12 - hi, r_lo = 12 - lo;
  return suited ? r_hi * 13 + r_lo : r_lo * 13 + r_hi;
}

HandClass HandClass::from_grid_index(int index) {
  int row = index / 13, col = index % 13;
  int r1 = 12 - row, r2 = 12 - col;
  if (row == col) return make(r1, r2, false);
  if (row < col) return make(r1, r2, true);
  return make(r1, r2, false);
}

int HandClass::num_combos() const { return is_pair() ? 6 : suited ? 4 : 12; }

std::vector<int> HandClass::combos() const {
  std::vector<int> out;
  for (int s1 = 0; s1 < 4; s1++)
    for (int s2 = 0; s2 < 4; s2++) {
      int a = make_card(hi, s1), b = make_card(lo, s2);
      if (a == b) continue;
      bool ok = is_pair() ? s1 < s2 : suited ? s1 == s2 : s1 != s2;
      if (ok) out.push_back(combo_index(a, b));
    }
  return out;
}

// ---------------------------------------------------------------- evaluator
// eval.rs:104-198.
static inline uint32_t high_bit(uint32_t x) { return 31u - (uint32_t)__builtin_clz(x); }

static inline uint32_t top_bits(uint32_t x, uint32_t n) {
  uint32_t out = 0;
  for (uint32_t i = 0; i < n; i++) {
    if (x == 0) break;
    uint32_t b = 1u << high_bit(x);
    out |= b;
    x ^= b;
  }
  return out;
}

// Returns the straight's high rank, or -1.
static inline int straight_high(uint32_t ranks) {
  const uint32_t WHEEL = 0x100F;  // A 5 4 3 2
  uint32_t run = ranks & (ranks << 1) & (ranks << 2) & (ranks << 3) & (ranks << 4);
  if (run != 0) return (int)high_bit(run);
  if ((ranks & WHEEL) == WHEEL) return 3;
  return -1;
}

enum { HIGH_CARD = 0, PAIR, TWO_PAIR, TRIPS, STRAIGHT, FLUSH, FULL_HOUSE, QUADS, STRAIGHT_FLUSH };

static inline uint32_t value_of(uint32_t cat, uint32_t payload) { return (cat << 26) | payload; }

uint32_t evaluate_mask(uint64_t mask) {
  uint32_t s0 = (uint32_t)(mask & 0x1FFF);
  uint32_t s1 = (uint32_t)((mask >> 16) & 0x1FFF);
  uint32_t s2 = (uint32_t)((mask >> 32) & 0x1FFF);
  uint32_t s3 = (uint32_t)((mask >> 48) & 0x1FFF);
  const uint32_t suits[4] = {s0, s1, s2, s3};
  for (uint32_t suited : suits) {
    if (__builtin_popcount(suited) >= 5) {
      int h = straight_high(suited);
      if (h >= 0) return value_of(STRAIGHT_FLUSH, (uint32_t)h);
      return value_of(FLUSH, top_bits(suited, 5));
    }
  }
  uint32_t any = s0 | s1 | s2 | s3;
  uint32_t two = (s0 & s1) | (s0 & s2) | (s0 & s3) | (s1 & s2) | (s1 & s3) | (s2 & s3);
  uint32_t three = (s0 & s1 & s2) | (s0 & s1 & s3) | (s0 & s2 & s3) | (s1 & s2 & s3);
  uint32_t four = s0 & s1 & s2 & s3;
  if (four != 0) {
    uint32_t q = high_bit(four);
    uint32_t kicker = top_bits(any & ~(1u << q), 1);
    return value_of(QUADS, (q << 13) | kicker);
  }
  if (three != 0) {
    uint32_t t = high_bit(three);
    uint32_t rest = two & ~(1u << t);
    if (rest != 0) {
      uint32_t p = high_bit(rest);
      return value_of(FULL_HOUSE, (t << 13) | (1u << p));
    }
  }
  {
    int h = straight_high(any);
    if (h >= 0) return value_of(STRAIGHT, (uint32_t)h);
  }
  if (three != 0) {
    uint32_t t = high_bit(three);
    uint32_t kickers = top_bits(any & ~(1u << t), 2);
    return value_of(TRIPS, (t << 13) | kickers);
  }
  if (__builtin_popcount(two) >= 2) {
    uint32_t pairs = top_bits(two, 2);
    uint32_t kicker = top_bits(any & ~pairs, 1);
    return value_of(TWO_PAIR, (pairs << 13) | kicker);
  }
  if (two != 0) {
    uint32_t p = high_bit(two);
    uint32_t kickers = top_bits(any & ~(1u << p), 3);
    return value_of(PAIR, (p << 13) | kickers);
  }
  return value_of(HIGH_CARD, top_bits(any, 5));
}

uint32_t evaluate_cards(const int* cards, int n) {
  uint64_t m = 0;
  for (int i = 0; i < n; i++) m |= eval_card_bit(cards[i]);
  return evaluate_mask(m);
}

// ---------------------------------------------------------------- menu
static std::string lower_trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  std::string t = s.substr(a, b - a);
  for (auto& c : t) c = (char)std::tolower((unsigned char)c);
  return t;
}

static bool parse_f64(const std::string& s0, double& out) {
  std::string s = lower_trim(s0);
  if (s.empty()) return false;
  char* end = nullptr;
  out = std::strtod(s.c_str(), &end);
  return end && *end == 0;
}

// menu.rs:26-50.
bool parse_bet_size(const std::string& s, BetSize& out) {
  std::string t = lower_trim(s);
  if (t == "a" || t == "allin" || t == "all-in" || t == "all in" || t == "shove") {
    out = BetSize{SIZE_ALLIN, 0.0};
    return true;
  }
  if (!t.empty() && t.back() == '%') {
    double v;
    if (!parse_f64(t.substr(0, t.size() - 1), v) || v <= 0.0) return false;
    out = BetSize{SIZE_POT, v / 100.0};
    return true;
  }
  if (!t.empty() && t.back() == 'x') {
    double v;
    if (!parse_f64(t.substr(0, t.size() - 1), v) || v <= 1.0) return false;
    out = BetSize{SIZE_MULT, v};
    return true;
  }
  return false;
}

static StreetSizes sizes_of(std::initializer_list<const char*> bet, std::initializer_list<const char*> raise) {
  StreetSizes s;
  for (auto b : bet) {
    BetSize x;
    parse_bet_size(b, x);
    s.bet.push_back(x);
  }
  for (auto r : raise) {
    BetSize x;
    parse_bet_size(r, x);
    s.raise.push_back(x);
  }
  return s;
}

PostflopMenu PostflopMenu::defaults() {
  PostflopMenu m;
  m.flop = sizes_of({"33%", "75%"}, {"3x"});
  m.turn = sizes_of({"50%", "100%"}, {"3x"});
  m.river = sizes_of({"50%", "100%"}, {"3x"});
  m.max_raises = 3;
  m.add_allin_threshold = 1.5;
  m.force_allin_threshold = 0.15;
  m.merge_threshold = 0.1;
  return m;
}

const StreetSizes& PostflopMenu::street(Street s) const {
  switch (s) {
    case TURN: return turn;
    case RIVER: return river;
    default: return flop;
  }
}

// Rust `f64::round() as i64`: C round() is half away from zero; the casts
// here stay in range.
static inline Chips round_chips(double x) { return (Chips)std::round(x); }

// finalize_tagged (menu.rs:355-392).
static std::vector<std::pair<Chips, size_t>> finalize_tagged(const Situation& sit,
                                                             std::vector<std::pair<Chips, size_t>> amounts,
                                                             double force_allin, double merge) {
  Chips lo = std::min(sit.min_raise_to, sit.max_to);
  Chips pot_after_call = sit.pot + sit.to_call;
  std::vector<std::pair<Chips, size_t>> v;
  for (auto& at : amounts) {
    Chips a = std::max(lo, std::min(at.first, sit.max_to));  // clamp(lo, max_to), lo <= max_to
    Chips new_pot = pot_after_call + 2 * (a - sit.current_bet);
    Chips threshold = round_chips((double)new_pot * force_allin);
    std::pair<Chips, size_t> x = (sit.max_to - a <= threshold) ? std::make_pair(sit.max_to, at.second)
                                                                 : std::make_pair(a, at.second);
    if (x.first > sit.current_bet) v.push_back(x);
  }
  std::sort(v.begin(), v.end());
  // dedup_by_key(|x| x.0): keep the first of each run of equal amounts.
  std::vector<std::pair<Chips, size_t>> d;
  for (auto& x : v)
    if (d.empty() || d.back().first != x.first) d.push_back(x);
  v = d;
  if (merge > 0.0 && v.size() > 1) {
    auto ratio = [&](Chips a) { return (double)(a - sit.current_bet) / (double)pot_after_call; };
    std::vector<std::pair<Chips, size_t>> kept;
    for (auto it = v.rbegin(); it != v.rend(); ++it) {
      if (!kept.empty() && (1.0 + ratio(kept.back().first)) / (1.0 + ratio(it->first)) < 1.0 + merge) continue;
      kept.push_back(*it);
    }
    std::reverse(kept.begin(), kept.end());
    v = kept;
  }
  return v;
}

// postflop_categorized (menu.rs:264-308), actions only.
std::vector<Action> postflop_actions(const Situation& sit, const PostflopMenu& menu) {
  std::vector<Action> out;
  if (sit.to_call > 0) {
    out.push_back(Action{FOLD, 0});
    out.push_back(Action{CALL, 0});
  } else {
    out.push_back(Action{CHECK, 0});
  }
  if (!sit.can_raise() || sit.num_raises >= menu.max_raises) return out;
  const StreetSizes& sizes = menu.street(sit.street);
  const std::vector<BetSize>& list = sit.current_bet == 0 ? sizes.bet : sizes.raise;
  double pot_after_call = (double)(sit.pot + sit.to_call);
  std::vector<std::pair<Chips, size_t>> amounts;
  for (size_t i = 0; i < list.size(); i++) {
    const BetSize& size = list[i];
    Chips to;
    if (size.kind == SIZE_POT) {
      to = sit.current_bet + round_chips(size.value * pot_after_call);
    } else if (size.kind == SIZE_MULT) {
      if (sit.current_bet == 0) continue;
      to = round_chips(size.value * (double)sit.current_bet);
    } else {
      to = sit.max_to;
    }
    amounts.push_back({to, i});
  }
  if (menu.add_allin_threshold > 0.0 &&
      (double)(sit.max_to - sit.current_bet) <= menu.add_allin_threshold * pot_after_call)
    amounts.push_back({sit.max_to, list.size()});
  auto fin = finalize_tagged(sit, amounts, menu.force_allin_threshold, menu.merge_threshold);
  for (auto& x : fin) out.push_back(Action{RAISE, x.first});
  return out;
}

// ---------------------------------------------------------------- ranges
// Pattern (range.rs:156-199) and expand_token (range.rs:201-238).
struct Pattern {
  int hi, lo;
  int suited;  // -1 = both
};

static bool parse_pattern(const std::string& s, Pattern& p) {
  if (s.size() < 2 || s.size() > 3) return false;
  int r1 = parse_rank(s[0]), r2 = parse_rank(s[1]);
  if (r1 < 0 || r2 < 0) return false;
  int hi = r1 >= r2 ? r1 : r2, lo = r1 >= r2 ? r2 : r1;
  int suited = -1;
  if (s.size() == 3) {
    char c = (char)std::tolower((unsigned char)s[2]);
    if (c == 's' && hi != lo) suited = 1;
    else if (c == 'o' && hi != lo) suited = 0;
    else return false;
  }
  p = Pattern{hi, lo, suited};
  return true;
}

static void pattern_classes(const Pattern& p, std::vector<HandClass>& out) {
  if (p.hi == p.lo) {
    out.push_back(HandClass::make(p.hi, p.lo, false));
    return;
  }
  if (p.suited >= 0) {
    out.push_back(HandClass::make(p.hi, p.lo, p.suited == 1));
  } else {
    out.push_back(HandClass::make(p.hi, p.lo, true));
    out.push_back(HandClass::make(p.hi, p.lo, false));
  }
}

static std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

static bool expand_token(const std::string& tok, std::vector<int>& out) {
  std::string lower = tok;
  for (auto& c : lower) c = (char)std::tolower((unsigned char)c);
  out.clear();
  if (lower == "any" || lower == "random" || lower == "all") {
    for (int i = 0; i < 1326; i++) out.push_back(i);
    return true;
  }
  if (tok.size() == 4) {
    std::vector<int> cards;
    if (parse_cards(tok, cards)) {
      if (cards[0] == cards[1]) return false;
      out.push_back(combo_index(cards[0], cards[1]));
      return true;
    }
  }
  std::vector<Pattern> patterns;
  size_t dash = tok.find('-');
  if (dash != std::string::npos) {
    Pattern pa, pb;
    if (!parse_pattern(trim(tok.substr(0, dash)), pa) || !parse_pattern(trim(tok.substr(dash + 1)), pb)) return false;
    if (pa.hi == pa.lo && pb.hi == pb.lo) {
      int lo = std::min(pa.hi, pb.hi), hi = std::max(pa.hi, pb.hi);
      for (int r = lo; r <= hi; r++) patterns.push_back(Pattern{r, r, -1});
    } else if (pa.hi == pb.hi && pa.suited == pb.suited && pa.hi != pa.lo && pb.hi != pb.lo) {
      int lo = std::min(pa.lo, pb.lo), hi = std::max(pa.lo, pb.lo);
      for (int l = lo; l <= hi; l++) patterns.push_back(Pattern{pa.hi, l, pa.suited});
    } else {
      return false;
    }
  } else if (!tok.empty() && tok.back() == '+') {
    Pattern p;
    if (!parse_pattern(trim(tok.substr(0, tok.size() - 1)), p)) return false;
    if (p.hi == p.lo) {
      for (int r = p.hi; r <= 12; r++) patterns.push_back(Pattern{r, r, -1});
    } else {
      for (int l = p.lo; l < p.hi; l++) patterns.push_back(Pattern{p.hi, l, p.suited});
    }
  } else {
    Pattern p;
    if (!parse_pattern(tok, p)) return false;
    patterns.push_back(p);
  }
  for (auto& p : patterns) {
    std::vector<HandClass> cls;
    pattern_classes(p, cls);
    for (auto& c : cls)
      for (int i : c.combos()) out.push_back(i);
  }
  return true;
}

// Range::from_str (range.rs:240-264).
bool parse_range(const std::string& s, std::vector<float>& out, std::string* err) {
  out.assign(1326, 0.0f);
  size_t start = 0;
  while (start <= s.size()) {
    size_t comma = s.find(',', start);
    std::string raw = trim(s.substr(start, comma == std::string::npos ? std::string::npos : comma - start));
    start = comma == std::string::npos ? s.size() + 1 : comma + 1;
    if (raw.empty()) continue;
    std::string tok = raw;
    float w = 1.0f;
    size_t colon = raw.find(':');
    if (colon != std::string::npos) {
      tok = trim(raw.substr(0, colon));
      std::string ws = trim(raw.substr(colon + 1));
      char* end = nullptr;
      w = std::strtof(ws.c_str(), &end);
      if (ws.empty() || !end || *end != 0) {
        if (err) *err = "invalid weight in " + raw;
        return false;
      }
    }
    std::vector<int> combos;
    if (!expand_token(tok, combos)) {
      if (err) *err = "invalid token " + tok;
      return false;
    }
    for (int c : combos) out[c] = w;
  }
  return true;
}

}  // namespace oracle
