// Device plan of one traversal: POD task records shared by the host planner
// (engine.cu) and the kernels (kernels.cu).
//
// A traversal for traverser p over a subtree is level-synchronous:
//   down levels  — opponent nodes split the opponent reach by their
//                  strategy (regret matching + strategy-sum update in CFR
//                  mode), chance nodes fan the reach out per dealt card;
//   terminals    — fold and showdown values of every live terminal, one
//                  warp per group of up to 32 terminals;
//   up levels    — deepest first: traverser nodes combine child values
//                  (and update regrets), opponent nodes and chance nodes sum.
// Reach rows live in "slots" (a traverser node's children share its slot);
// value rows are indexed by node id. Every row has HP floats (hands padded
// to a multiple of 8, padding kept at zero).
#pragma once

#include <cstdint>

namespace dcfr {

constexpr int VEC = 4;             // hands per thread in the row kernels (float4)
constexpr int ROW_MAX_THREADS = 352;  // row-kernel block: a thread per 4 hands, whole warps (1328 hands max)
constexpr int MAX_ACTIONS = 16;
constexpr int TERM_WARPS = 4;      // warps per terminal-kernel block
constexpr int TERM_CHUNK = 32;     // sweep steps staged per cp.async batch
constexpr uint32_t NONE32 = 0xFFFFFFFFu;

enum DownKind : uint32_t { D_OPP_SPLIT = 0, D_CHANCE_SPLIT = 1 };
enum UpKind : uint32_t { U_OWN = 0, U_OPP_SUM = 1, U_CHANCE_SUM = 2 };
enum TermKind : uint32_t { T_FOLD_SCALAR = 0, T_FOLD_BATCH = 1, T_SHOWDOWN_SCALAR = 2, T_SHOWDOWN_BATCH = 3 };
enum ModeId : int { M_CFR = 0, M_BR = 1, M_AVG = 2 };

struct DownTask {
  uint32_t kind;
  uint32_t in_slot;   // reach slot of the node
  uint32_t out_slot;  // slot of the first child (children's slots are consecutive)
  uint32_t nchild;
  uint64_t store;     // opponent split: float offset of the node's block
  uint32_t cards;     // chance split: offset of the children's cards in chance_cards;
                      // opponent split: the node's scale slot (compressed storage)
  float factor;       // chance split: reach multiplier
};

struct UpTask {
  uint32_t kind;
  uint32_t slot;        // reach slot of the node (liveness)
  uint32_t node;        // value row
  uint32_t child;       // first child's node id (value rows are consecutive)
  uint32_t nchild;
  uint32_t child_slot;  // first child's slot (opponent / chance nodes)
  uint64_t store;       // traverser node: float offset of its block
  uint32_t cards;       // chance: offset of the children's cards; decision node:
                        // its scale slot (compressed storage)
  uint32_t iso_first;   // chance: first isomorphic reference
  uint32_t iso_count;
  uint32_t pad;
};

// Fused river subtree: the down and up tasks of all its decision nodes,
// processed by one block (down: BFS order, LEVEL_BREAK on a level's first
// task; up: deepest level first).
struct FusedTree {
  uint32_t down_first, down_count;
  uint32_t up_first, up_count;
};
constexpr uint32_t LEVEL_BREAK = 0x100u;  // in DownTask::kind
constexpr uint32_t KIND_MASK = 0xFFu;

struct IsoRefD {
  uint16_t ci;    // canonical child index
  uint8_t pair;   // suit pair (0..5)
  uint8_t pad;
};

struct TermLane {
  uint32_t slot;  // reach slot
  uint32_t row;   // value row (node id)
  uint32_t frow;  // paired fold's value row, or NONE32
  uint32_t pad;
  double a;       // fold payoff / showdown win
  double b;       // showdown lose
  double c;       // showdown tie
  double d;       // paired fold payoff
};

// One warp's work in the terminal kernel: a fold group, or one of the
// passes of a showdown group (ascending win part, descending lose part,
// paired fold). wgroup indexes the per-launch win/lose scratch and counter.
enum TermRole : uint32_t { R_FOLD = 0, R_ASC = 1, R_DESC = 2, R_PAIRED = 3 };
struct TermTask {
  uint32_t role;
  uint32_t group;
  uint32_t wgroup;
  uint32_t pad;
};
constexpr int MAX_WAVE_TASKS = 1024;   // warps per terminal launch
constexpr int MAX_WAVE_GROUPS = 384;   // showdown groups per terminal launch

struct TermGroup {
  uint32_t kind;
  uint32_t board;  // showdown strength table
  uint32_t first;  // first lane in the lane array
  uint32_t count;  // lanes used (1..32)
};

// Strength-table entry (eval::Entry, crates/solver/src/eval.rs:11-18).
struct EntryD {
  uint32_t strength;
  uint16_t idx;
  uint8_t c1, c2;
};

struct DiscountD {
  float pos, neg, strat;
  int reach_weighted;
};

// One decision node's storage block for transfers to and from the
// reference's layout (HostStorage, crates/solver/src/storage.rs): its
// [rows][hp] block at element `dev` of the device storage, and its
// [rows][n] block at element `host` of the reference layout, counted from
// the start of the transfer chunk that holds it.
struct StorageBlockD {
  uint64_t dev, host;
  uint32_t rows, n, hp, pad;
};

// Fast-precision terminal evaluation (terminal_fast.cu): one task per live
// terminal; a showdown task also writes its paired fold's row.
struct FastTask {
  uint32_t kind;   // TermKind
  uint32_t board;  // layout index: showdown board, or the fold layout
  uint32_t slot;   // reach slot
  uint32_t row;    // value row (node id)
  uint32_t frow;   // paired fold's value row, or NONE32
  uint32_t pad[3];
  double a, b, c, d;  // as TermLane
};

// A depth-limited solve's leaf in one traversal: the leaf's ordinal, the
// reach slot arriving at it and the value row (node id) it fills, and the
// state entering the network (pot and effective stack in chips).
struct LeafTask {
  uint32_t leaf;
  uint32_t slot;
  uint32_t row;
  uint32_t pad;
  float pot;
  float stack;
};

// Longest opponent hand list evaluated warp per terminal; longer lists use
// the block-wide scan of fast_terminal_kernel (measured: the block kernel is
// faster at 1128 hands, the warp kernel at 470).
constexpr int WARP_TERMINAL_MAX_HANDS = 768;
// A maximal run of fast terminal tasks on one layout. The warp terminal
// kernel (terminal_fast.cu) stages a run's layout in shared memory once per
// block whose task range meets the run.
struct TermUnit {
  uint32_t layout;  // FastTask::board of every task in the run
  uint32_t first;   // first task
  uint32_t count;   // tasks
  uint32_t pad;
};

// A panel of the panel terminal kernel (terminal_panel.cu): `count` (1..T)
// consecutive fast terminal tasks, all on one layout and all showdowns or
// all folds.
struct PanelD {
  uint32_t first;   // first task
  uint32_t count;   // tasks
  uint32_t layout;  // FastTask::board of every task in the panel
  uint32_t pad;
};

// Per (layout, traverser) scan layout of the opponent's hands: segment 0
// lists them in ascending strength, segment 1+c lists those holding card c
// (ascending strength). seg[j] is the first element of segment j
// (seg[53] = 3 * count). Per traverser hand h, rec[h] = {w | s << 16,
// aw | as << 16, bw | bs << 16, a | b << 8 | present << 16}: w (s) counts the
// opponent hands weaker than (not stronger than) h, aw/as (bw/bs) index the
// same boundaries inside card a's (b's) segment.
constexpr int FAST_SEGS = 54;
constexpr int FAST_THREADS = 256;

// R is the row type: float for the solve, double for the FP64 best-response
// oracle (br64.cu).
template <typename R>
struct FastArgsT {
  const R* reach;
  R* vals;
  const uint32_t* alive;
  const uint16_t* cat;   // [(layout*2+p)][cstride] opponent hand per element
  const uint16_t* seg;   // [(layout*2+p)][FAST_SEGS]
  const uint4* rec;      // [(layout*2+p)][tstride]
  const uint32_t* same;  // traverser hand -> identical opponent hand (or NONE32)
  int cstride;
  int tstride;
  int emax;              // elements per thread (odd) for the largest layout
  int n[2];
  int hp[2];
  int stride;
  int p;
};
using FastArgs = FastArgsT<float>;
using FastArgs64 = FastArgsT<double>;

// Arguments of the row kernels (down/up levels) of one traversal.
struct RowArgs {
  float* regrets;
  float* sums;
  // 16-bit compressed storage (set instead of regrets / sums): i16 regrets,
  // u16 sums, one f32 scale of each per decision node (its ordinal).
  int16_t* rq;
  uint16_t* sq;
  float* rscale;
  float* sscale;
  int compressed;
  float* reach;
  float* vals;
  uint32_t* alive;
  const uint8_t* hc1[2];  // hand cards, padded to hp with 255
  const uint8_t* hc2[2];
  const uint16_t* perm;   // [(q*6+pair)*stride + h]
  const uint8_t* chance_cards;
  const IsoRefD* iso;
  const DiscountD* disc;
  int n[2];
  int hp[2];
  int stride;
  int p;
};

// Arguments of the FP64 best-response kernels (br64.cu): double reach and
// value rows, the f32 strategy sums.
struct Row64Args {
  const float* sums;
  const uint16_t* sq;     // compressed storage: u16 sums and per-node scales (sums is null)
  const float* sscale;
  double* reach;
  double* vals;
  uint32_t* alive;
  const uint8_t* hc1[2];
  const uint8_t* hc2[2];
  const uint16_t* perm;
  const uint8_t* chance_cards;
  const IsoRefD* iso;
  int n[2];
  int hp[2];
  int stride;
  int p;
};

// Arguments of the terminal kernel.
struct TermArgs {
  const float* reach;
  float* vals;
  const uint32_t* alive;
  float* warp_scratch;          // per warp: Rp [pstride+1][32], O [stride][32]
  size_t warp_scratch_floats;
  double* group_scratch;        // per showdown group: win and lose parts [2][nmax][32]
  uint32_t* counters;           // per showdown group: passes finished
  const EntryD* tables;
  const uint32_t* table_count;
  const uint32_t* progs;        // [((board*2+p)*3+dir)][pstride] sweep programs
  const uint32_t* prog_count;   // steps per program (a multiple of TERM_CHUNK)
  const uint32_t* posmap;       // [((board*2+p)*3+dir)][tstride] opponent hand -> step
  const uint32_t* fold_prog[2]; // each player's hands in hand order as steps
  const uint2* emit_rec[2];     // per hand: blocker rows word, identical opponent hand
  int pstride;
  const uint8_t* hc1[2];
  const uint8_t* hc2[2];
  const uint32_t* same[2];
  int n[2];
  int hp[2];
  int stride;
  int tstride;
  int nmax;
  int p;
};

}  // namespace dcfr
