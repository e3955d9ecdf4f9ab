/*
 * dcfr.h — C ABI of libdcfr, the B200 heads-up Discounted-CFR range-vs-range
 * postflop solver.
 *
 * The ABI mirrors the public API of the reference solver crate
 * (AhanDatta/Poker-Trainer, crates/solver/src/lib.rs): build a game from a
 * board, two 1326-combo ranges, a root betting state and bet menus; solve it
 * with DCFR; query per-node strategies, EVs, ranges and exploitability.
 * Every function returns an int status (DCFR_OK or a DCFR_ERR_* code); the
 * message of the last failure on the calling thread is dcfr_last_error().
 * All buffers are caller-allocated. There is no CPU fallback: a solver
 * handle owns one CUDA stream on the current device, and every iteration,
 * best response and query traversal runs in the library's sm_100a kernels.
 * One handle is used by one thread at a time.
 *
 * Card ids are rank*4+suit with ranks 2..A = 0..12 and suits c,d,h,s = 0..3
 * (crates/holdem/src/card.rs:46). Combo ids are hi*(hi-1)/2+lo over card ids
 * with hi > lo (crates/holdem/src/combo.rs:14-17).
 */
#ifndef DCFR_H
#define DCFR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DCFR_NUM_COMBOS 1326
#define DCFR_MAX_SIZES 8

/* Status codes. The first four mirror SolverError
 * (crates/solver/src/lib.rs:186-192). */
enum {
  DCFR_OK = 0,
  DCFR_ERR_EMPTY_RANGE = 1,   /* SolverError::EmptyRange(player) */
  DCFR_ERR_INVALID_BOARD = 2, /* SolverError::InvalidBoard */
  DCFR_ERR_TOO_LARGE = 3,     /* SolverError::TooLarge{needed, limit} */
  DCFR_ERR_BAD_PATH = 4,      /* SolverError::BadPath */
  DCFR_ERR_INVALID_ARG = 5,   /* malformed config, NULL pointer, short buffer */
  DCFR_ERR_CUDA = 6,          /* a CUDA runtime call failed */
  DCFR_ERR_OUT_OF_MEMORY = 7, /* device memory exhausted */
  DCFR_ERR_UNSUPPORTED = 8,   /* option not built for this solver kind */
  DCFR_ERR_DEVICE_TIMEOUT = 9 /* a bounded device-side wait gave up */
};

/* Streets (holdem::Street, crates/holdem/src/game.rs:19-25). */
enum { DCFR_PREFLOP = 0, DCFR_FLOP = 1, DCFR_TURN = 2, DCFR_RIVER = 3 };

/* Bet size kinds (holdem::menu::BetSize, crates/holdem/src/menu.rs:16-24). */
enum { DCFR_SIZE_POT = 0, DCFR_SIZE_MULT = 1, DCFR_SIZE_ALLIN = 2 };

/* Action kinds (holdem::Action, crates/holdem/src/game.rs:76-82). */
enum { DCFR_FOLD = 0, DCFR_CHECK = 1, DCFR_CALL = 2, DCFR_RAISE = 3 };

/* Storage modes (StorageMode, crates/solver/src/storage.rs:79-85). */
enum { DCFR_STORAGE_F32 = 0, DCFR_STORAGE_COMPRESSED = 1, DCFR_STORAGE_AUTO = 2 };

/* GpuPrecision (crates/solver/src/gpu/mod.rs:51-63). FAST (the default, as
 * in the reference) evaluates terminals with exact 64-bit fixed-point sums of
 * the f32 reach, which agree with the CPU's sequential f64 sums except for
 * rare one-rounding-step differences; EXACT sweeps in the CPU's f64
 * operation order and is bit-identical to the CPU solver. */
enum { DCFR_PRECISION_FAST = 0, DCFR_PRECISION_EXACT = 1 };

/* Chance modes (ChanceMode, crates/solver/src/tree.rs:128-136). SAMPLED deals
 * a stratified sample of chance_turn turn cards and chance_river river cards
 * per chance node (sample_cards, crates/solver/src/sampling.rs:9-54), drawn
 * from rand 0.9's StdRng seeded with chance_seed; all-in runouts stay
 * exact. */
enum { DCFR_CHANCE_EXACT = 0, DCFR_CHANCE_SAMPLED = 1 };

/* Traversal modes (cfr::Mode, crates/solver/src/cfr.rs:248-256). */
enum { DCFR_MODE_CFR = 0, DCFR_MODE_BEST_RESPONSE = 1, DCFR_MODE_AVERAGE = 2 };

/* One bet size: kind DCFR_SIZE_*, value = pot fraction (0.75 for 75%) or
 * raise multiple (3.0 for 3x); ignored for all-in. */
typedef struct dcfr_bet_size {
  int32_t kind;
  int32_t _pad;
  double value;
} dcfr_bet_size;

/* StreetSizes (crates/holdem/src/menu.rs:87-91). */
typedef struct dcfr_street_sizes {
  int32_t n_bet;
  int32_t n_raise;
  dcfr_bet_size bet[DCFR_MAX_SIZES];
  dcfr_bet_size raise[DCFR_MAX_SIZES];
} dcfr_street_sizes;

/* PostflopMenu (crates/holdem/src/menu.rs:102-117). */
typedef struct dcfr_menu {
  dcfr_street_sizes flop;
  dcfr_street_sizes turn;
  dcfr_street_sizes river;
  uint32_t max_raises;
  uint32_t _pad;
  double add_allin_threshold;
  double force_allin_threshold;
  double merge_threshold;
} dcfr_menu;

/* BettingState (crates/solver/src/tree.rs:19-34). Player 0 is out of
 * position. */
typedef struct dcfr_betting_state {
  int32_t street;
  int32_t to_act;
  int64_t pot;
  int64_t commit[2];
  int64_t stack[2];
  int64_t current_bet;
  int64_t last_raise_inc;
  uint32_t num_raises;
  uint8_t needs[2];
  uint8_t _pad[2];
} dcfr_betting_state;

/* DcfrParams (crates/solver/src/cfr.rs:48-63). beta_clip != 0 means
 * beta = None (negative regrets clipped to zero, DCFR+). */
typedef struct dcfr_params {
  double alpha;
  double beta;
  double gamma;
  int32_t beta_clip;
  int32_t restart_average;
  int32_t unweighted_average;
  int32_t _pad;
} dcfr_params;

/* SolveConfig (crates/solver/src/lib.rs:74-105). Ranges are inline
 * 1326-entry weight vectors indexed by combo id. keep[p] lists up to
 * n_keep[p] combo ids that pruning must never drop. */
typedef struct dcfr_config {
  uint8_t board[5];
  uint8_t _pad0[3];
  int32_t board_len;
  int32_t _pad1;
  float ranges[2][DCFR_NUM_COMBOS];
  dcfr_betting_state root;
  dcfr_menu menu;
  int32_t has_future_menu;
  int32_t _pad2;
  dcfr_menu future_menu;
  int64_t big_blind;
  float prune;
  int32_t n_keep[2];
  int32_t _pad3;
  uint16_t keep[2][DCFR_NUM_COMBOS];
  uint64_t max_memory_bytes;
  double rake_rate;
  double rake_cap;
  int32_t storage;
  int32_t isomorphism;
  dcfr_params dcfr;
  int32_t precision; /* DCFR_PRECISION_* (Solver::use_gpu(precision), lib.rs:508-530) */
  int32_t chance;    /* DCFR_CHANCE_* (SolveConfig::chance, lib.rs:88) */
  int32_t chance_turn;
  int32_t chance_river;
  uint64_t chance_seed;
} dcfr_config;

/* TreeStats (crates/solver/src/tree.rs:248-257). */
typedef struct dcfr_tree_stats {
  uint64_t player_nodes;
  uint64_t chance_nodes;
  uint64_t terminal_nodes;
  uint64_t storage_cells;
  int32_t compressed;
  int32_t _pad;
  uint64_t memory_bytes;
} dcfr_tree_stats;

/* SolveOptions (crates/solver/src/lib.rs:137-147). */
typedef struct dcfr_solve_options {
  uint32_t max_iterations;
  uint32_t check_every;
  double target_exploitability_pct;
} dcfr_solve_options;

/* Progress (crates/solver/src/lib.rs:174-184). */
typedef struct dcfr_progress {
  uint32_t iteration;
  uint32_t max_iterations;
  double exploitability;
  double exploitability_pct;
  int32_t finished;
  int32_t _pad;
} dcfr_progress;

/* Called after every exploitability check; returning 0 cancels the solve
 * (the on_progress closure of Solver::solve, lib.rs:475). */
typedef int (*dcfr_progress_cb)(const dcfr_progress* progress, void* user);

/* A path step (Step, crates/solver/src/lib.rs:212-217): kind 0 = action
 * (action_kind DCFR_FOLD..DCFR_RAISE, amount = raise-to chips), kind 1 =
 * dealt card. */
typedef struct dcfr_step {
  int32_t kind;
  int32_t action_kind;
  int64_t amount;
  uint8_t card;
  uint8_t _pad[7];
} dcfr_step;

typedef struct dcfr_action {
  int32_t kind;
  int32_t _pad;
  int64_t amount;
} dcfr_action;

/* Header of NodeInfo (crates/solver/src/lib.rs:220-240); the arrays are
 * written by dcfr_query into caller buffers sized from dcfr_query_sizes. */
typedef struct dcfr_node_info {
  int32_t player;
  int32_t num_actions;
  int32_t num_hands;
  int32_t _pad;
  double reach_fraction[2];
  int64_t pot;
  int64_t invest[2];
} dcfr_node_info;

typedef struct dcfr_solver dcfr_solver;

/* Message of the last failed call on this thread ("" if none). */
const char* dcfr_last_error(void);

/* SolveConfig::new defaults (lib.rs:110-134) with the default PostflopMenu
 * (menu.rs:119-133): exact runouts, no rake, Auto storage, isomorphism on,
 * 8 GiB limit, DcfrParams::default (cfr.rs:72-80). board/ranges/root are
 * left zeroed for the caller. */
int dcfr_config_init(dcfr_config* cfg);

/* Solver::estimate (lib.rs:355-362): tree size without building it. */
int dcfr_estimate(const dcfr_config* cfg, dcfr_tree_stats* out);

/* Solver::new (lib.rs:365-396): builds the tree, the strength tables and
 * the device plan, and allocates device storage on the current device. */
int dcfr_create(const dcfr_config* cfg, dcfr_solver** out);
void dcfr_destroy(dcfr_solver* s);

/* Solver::solve_cancellable (lib.rs:482-494) over run_solve
 * (lib.rs:594-642): iterations, exploitability checks on the
 * next_check_gap schedule (lib.rs:158-172), cancellation checked before
 * every iteration. cancel and cb may be NULL. */
int dcfr_solve(dcfr_solver* s, const dcfr_solve_options* opts, const volatile int32_t* cancel,
               dcfr_progress_cb cb, void* user, dcfr_progress* out);

/* Runs exactly n DCFR iterations (cpu_iteration, lib.rs:577-585) with no
 * exploitability checks. Asynchronous on the handle's stream. */
int dcfr_iterate(dcfr_solver* s, uint32_t n);
/* Waits for the handle's stream. */
int dcfr_synchronize(dcfr_solver* s);

/* Solver::exploitability (lib.rs:462-464), chips. */
int dcfr_exploitability(dcfr_solver* s, double* out);
/* No counterpart in the reference: the FP64 best-response oracle. The same
 * exploitability as dcfr_exploitability (cfr.rs:482-502), with every reach
 * and value row of the two best-response traversals held in double on the
 * GPU (average strategies normalised in double from the f32 sums, terminal
 * sums exact in 64-bit fixed point, payoffs in double). best_response (may be
 * NULL) receives each player's best-response root value in chips. The first
 * call allocates the double rows on the device. */
int dcfr_exploitability_fp64(dcfr_solver* s, double* out, double best_response[2]);
/* No counterpart in the reference: a depth-limited flop solve. The tree of a
 * flop-root config ends at the turn deal, and every traversal values those
 * leaves with the leaf-value network `net` (dcfr_mlp_*, 2706 inputs, 2652
 * outputs, max batch at least leaves x 49): for each dealt card the network
 * gives every combo's EV in pots from both players' ranges, the board, pot
 * and stack, and the leaf sums them as a chance node sums its children.
 * Fast precision, no rake. net must outlive the solver; everything else
 * (dcfr_iterate, dcfr_solve, queries, exploitability of the depth-limited
 * game) works as for dcfr_create. */
typedef struct dcfr_mlp dcfr_mlp;
int dcfr_create_depth_limited(const dcfr_config* cfg, dcfr_mlp* net, dcfr_solver** out);
/* Offset, action count and hand count of the decision node at `path` in the
 * reference storage layout (Node::offset, tree.rs:200-204): its block in
 * dcfr_download_storage / dcfr_upload_storage arrays. */
int dcfr_node_storage(dcfr_solver* s, const dcfr_step* path, size_t n, uint64_t* offset, int32_t* num_actions,
                      int32_t* num_hands);
/* Overwrites the regrets and/or strategy sums (either may be NULL) of the
 * decision node at `path` from [num_actions][num_hands] blocks in the
 * reference layout; e.g. to evaluate a depth-limited solve's flop strategy
 * inside a full tree. */
int dcfr_write_node(dcfr_solver* s, const dcfr_step* path, size_t n, const float* regrets, const float* sums);
/* Solver::root_values (lib.rs:468-470): average-strategy EV of each player. */
int dcfr_root_values(dcfr_solver* s, double out[2]);
/* Solver::iterations, last_exploitability, stats, root_pot. */
int dcfr_iterations(const dcfr_solver* s, uint32_t* out);
int dcfr_last_exploitability(const dcfr_solver* s, double* out);
int dcfr_stats(const dcfr_solver* s, dcfr_tree_stats* out);
/* Number of suit pairs solved through isomorphism (lib.rs:416-418). */
int dcfr_isomorphic_pairs(const dcfr_solver* s, int32_t* out);

/* Solver::hands (hands.rs:15-30): number of hands of player p, and their
 * combo ids and root weights (either pointer may be NULL). */
int dcfr_hands(const dcfr_solver* s, int32_t p, uint16_t* combos, float* weights, int32_t* n);

/* Solver::is_decision / actions_at / query / ranges_after
 * (lib.rs:828-912). dcfr_query_sizes gives the array sizes of dcfr_query:
 * actions[num_actions], combos[num_hands], strategy/ev[num_actions*num_hands]
 * (action-major), reach[num_hands]. */
int dcfr_is_decision(dcfr_solver* s, const dcfr_step* path, size_t n, int32_t* out);
int dcfr_actions_at(dcfr_solver* s, const dcfr_step* path, size_t n, dcfr_action* actions, size_t cap,
                    size_t* count);
int dcfr_query_sizes(dcfr_solver* s, const dcfr_step* path, size_t n, int32_t* num_actions,
                     int32_t* num_hands);
int dcfr_query(dcfr_solver* s, const dcfr_step* path, size_t n, dcfr_node_info* info,
               dcfr_action* actions, uint16_t* combos, float* strategy, float* ev, float* reach);
int dcfr_ranges_after(dcfr_solver* s, const dcfr_step* path, size_t n, float out[2][DCFR_NUM_COMBOS]);

/* Storage in the reference layout (storage.rs:87-98; one action-major
 * block per decision node at Node::offset, tree.rs:200-204): len f32
 * regrets and len f32 strategy sums. Used to resume a solve elsewhere
 * (lib.rs:532-540) and by the parity tests. A solver with compressed
 * storage downloads its values decoded (load_regrets / load_strat,
 * storage.rs:226-268) and uploads only through the compressed call. The
 * f32 and compressed transfers remove (or restore) the device layout's
 * padding on the device and copy each chunk (at most 64 M values) straight
 * between the device and the caller's arrays; page-locked arrays
 * (cudaHostAlloc) take the fastest copies. A transfer allocates a device
 * staging buffer of up to 256 MB for its duration. */
int dcfr_storage_len(const dcfr_solver* s, uint64_t* len);
int dcfr_download_storage(dcfr_solver* s, float* regrets, float* sums, uint64_t len);
int dcfr_upload_storage(dcfr_solver* s, const float* regrets, const float* sums, uint64_t len);
/* Compressed storage (Storage::Compressed, storage.rs:92-97; chosen by
 * DCFR_STORAGE_COMPRESSED, or by DCFR_STORAGE_AUTO when the f32 tree would
 * exceed 1 GB, as StorageMode::Auto): len i16 regrets and len u16 strategy
 * sums in the reference layout, and per decision node slot (Node::slot,
 * tree.rs:463) one f32 regret scale and one f32 sum scale; the stored
 * values decode as regret * scale / 32767 and sum * scale / 65535. The
 * HostStorage::Compressed transfer of the reference's GPU engine
 * (gpu/engine.rs:292-425). */
int dcfr_storage_slots(const dcfr_solver* s, uint64_t* slots);
int dcfr_download_storage_compressed(dcfr_solver* s, int16_t* regrets, uint16_t* sums, float* regret_scale,
                                     float* sum_scale, uint64_t len, uint64_t slots);
int dcfr_upload_storage_compressed(dcfr_solver* s, const int16_t* regrets, const uint16_t* sums,
                                   const float* regret_scale, const float* sum_scale, uint64_t len, uint64_t slots);
/* Sets the iteration counter (after uploading storage from another run). */
int dcfr_set_iterations(dcfr_solver* s, uint32_t t);

/* One traversal from the root for traverser p with the opponent's root
 * weights (cfr::traverse, cfr.rs:259-262): mode DCFR_MODE_*; iteration t
 * picks the DCFR discount (Discount::new, cfr.rs:86-106) in CFR mode.
 * Writes the root value row (n_p floats) to out. */
int dcfr_traverse(dcfr_solver* s, int32_t p, int32_t mode, uint32_t t, float* out);

/* Number of kernel launches the library issued on this handle so far. */
int dcfr_kernel_launches(const dcfr_solver* s, uint64_t* out);

/* Device time of the last dcfr_iterate call, in milliseconds (CUDA events
 * on the handle's stream around the launches), and the algorithmic bytes
 * one DCFR iteration moves (20 B per storage cell plus one opponent-reach
 * row read and one value row write per node and traversal). */
int dcfr_last_iterate_ms(dcfr_solver* s, double* ms);
int dcfr_iteration_bytes(const dcfr_solver* s, double* bytes);

/* Kernel classes of one traversal: down levels (opponent and chance
 * splits), the terminal launch, up levels (own-node updates, opponent and
 * chance sums), and everything else (discount advance, row resets, the gaps
 * between graph launches). */
enum { DCFR_KERNEL_DOWN = 0, DCFR_KERNEL_TERMINAL = 1, DCFR_KERNEL_UP = 2, DCFR_KERNEL_OTHER = 3 };
#define DCFR_KERNEL_CLASSES 4

typedef struct dcfr_kernel_profile {
  uint32_t iterations;
  uint32_t _pad;
  uint64_t launches[DCFR_KERNEL_CLASSES]; /* kernel launches per class */
  double ms[DCFR_KERNEL_CLASSES];         /* summed device time per class */
  double bytes[DCFR_KERNEL_CLASSES];      /* compulsory bytes per class: rows read and
                                             written, storage read and written */
  double total_ms;                        /* first to last event */
} dcfr_kernel_profile;

/* Measurement hooks, no counterpart in the reference. dcfr_last_solve_ms:
 * device time of the last dcfr_solve in milliseconds (CUDA events on the
 * handle's stream at its start and end). dcfr_setup_profile: where the
 * handle's setup went, host wall clock in milliseconds: the game (tree,
 * hands, isomorphism) built on the host; hands and chance tables uploaded;
 * strength tables and terminal layouts built on the device; both traversal
 * plans built (on two host threads while the storage is allocated and
 * cleared on the device) and uploaded; reach and value rows allocated; all
 * of dcfr_create; and, when they happen, the
 * iteration graph's capture (first dcfr_iterate / dcfr_solve) and the
 * best-response and average graphs' (first exploitability or root values). */
typedef struct dcfr_setup_profile {
  double game_ms;
  double device_ms;
  double tables_ms;
  double plans_ms;
  double rows_ms;
  double create_ms;
  double iteration_graph_ms;
  double eval_graphs_ms;
} dcfr_setup_profile;
int dcfr_last_solve_ms(const dcfr_solver* s, double* ms);
int dcfr_setup_profile_get(const dcfr_solver* s, dcfr_setup_profile* out);

/* Measurement hook, no counterpart in the reference: the terminal kernel
 * this handle's f32 traversals launch (DCFR_TERMINAL_*; GROUP: two warps per
 * terminal), and for the panel kernel the terminals evaluated together per
 * panel (0 otherwise). */
enum {
  DCFR_TERMINAL_PANEL = 0,
  DCFR_TERMINAL_WARP = 1,
  DCFR_TERMINAL_BLOCK = 2,
  DCFR_TERMINAL_EXACT = 3,
  DCFR_TERMINAL_GROUP = 4
};
int dcfr_terminal_kernel(const dcfr_solver* s, int32_t* kernel, int32_t* terminals_per_panel);

/* Measurement hook, no counterpart in the reference: runs `iterations` DCFR
 * iterations (they advance the solve exactly as dcfr_iterate's) from a second
 * captured graph that also records a CUDA event on the handle's stream at
 * every class boundary, and returns the per-class totals. */
int dcfr_iterate_profiled(dcfr_solver* s, uint32_t iterations, dcfr_kernel_profile* out);

/* ---- Batched river solves (no counterpart in the reference) ----------
 * Many independent river spots (5-card board, river root, fast precision,
 * one shared DcfrParams) solved together: each DCFR iteration of every spot
 * is the same as a single dcfr_create/dcfr_iterate solve of that spot, done
 * by one persistent kernel per block of iterations launched from a captured
 * CUDA graph; spots of uneven tree size are taken from a work counter,
 * longest first. */
typedef struct dcfr_batch dcfr_batch;

/* Launch shape of the batched kernel, chosen by dcfr_batch_autotune. */
typedef struct dcfr_batch_tuning {
  int32_t warps;                  /* warps per block (each evaluates terminals) */
  int32_t blocks_per_sm;          /* resident blocks per SM (grid = SMs x this) */
  uint32_t iterations_per_launch; /* iterations of a spot per persistent launch */
  int32_t longest_first;          /* 1: spots taken by decreasing work; 0: input order */
  int32_t candidates;             /* autotune: candidates timed */
  int32_t _pad;
  double trial_ms;                /* autotune: the best candidate's time */
} dcfr_batch_tuning;

int dcfr_batch_create(const dcfr_config* cfgs, int32_t count, dcfr_batch** out);
void dcfr_batch_destroy(dcfr_batch* b);
/* n DCFR iterations of every spot (cpu_iteration, lib.rs:577-585, per spot). */
int dcfr_batch_iterate(dcfr_batch* b, uint32_t n);
/* Per-spot exploitability in chips (cfr.rs:482-502); out has count entries. */
int dcfr_batch_exploitability(dcfr_batch* b, double* out);
/* One spot's storage in the reference layout (as dcfr_download_storage). */
int dcfr_batch_storage_len(const dcfr_batch* b, int32_t spot, uint64_t* len);
int dcfr_batch_download_storage(dcfr_batch* b, int32_t spot, float* regrets, float* sums, uint64_t len);
/* Times every launch shape that fits on trial_iterations iterations from a
 * snapshot of the storage (restored after each trial) and keeps the fastest. */
int dcfr_batch_autotune(dcfr_batch* b, uint32_t trial_iterations, dcfr_batch_tuning* out);
int dcfr_batch_get_tuning(const dcfr_batch* b, dcfr_batch_tuning* out);
int dcfr_batch_set_tuning(dcfr_batch* b, const dcfr_batch_tuning* t);
/* Device time of the last dcfr_batch_iterate (CUDA events on its stream),
 * iterations done, and kernel launches issued. */
int dcfr_batch_last_iterate_ms(const dcfr_batch* b, double* ms);
int dcfr_batch_iterations(const dcfr_batch* b, uint32_t* out);
int dcfr_batch_kernel_launches(const dcfr_batch* b, uint64_t* out);
/* Algorithmic bytes of one iteration of every spot (as dcfr_iteration_bytes,
 * summed over spots). */
int dcfr_batch_iteration_bytes(const dcfr_batch* b, double* bytes);

/* ---- Leaf-value network (no counterpart in the reference) ---------------
 * An MLP (in_dim -> `layers` hidden layers of width `hidden`, GELU -> out_dim)
 * trained and evaluated with the library's BF16 tcgen05 GEMM (FP32
 * accumulation, FP32 master weights, Adam). All arrays passed as x, y,
 * target and mask are device memory, row-major, one sample per row. */
int dcfr_mlp_create(int32_t in_dim, int32_t hidden, int32_t layers, int32_t out_dim, int32_t max_batch, uint64_t seed,
                    dcfr_mlp** out);
void dcfr_mlp_destroy(dcfr_mlp* n);
/* Parameter count of the flat layout (per layer W_t[out_pad][in_pad], then
 * per layer b[out_pad]; every dimension padded to a multiple of 128). */
int dcfr_mlp_num_params(const dcfr_mlp* n, uint64_t* out);
int dcfr_mlp_get_params(const dcfr_mlp* n, float* host);
int dcfr_mlp_set_params(dcfr_mlp* n, const float* host);
/* y[M][out_dim] = network(x[M][in_dim]). */
int dcfr_mlp_forward(dcfr_mlp* n, const float* x, int32_t m, float* y);
/* Loss sum(mask * (y - target)^2) / sum(mask) (mask may be NULL: all ones)
 * and its gradient in the flat layout (grads_host may be NULL). */
int dcfr_mlp_gradients(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t m, float* loss,
                       float* grads_host);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on that loss. */
int dcfr_mlp_train_step(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t m, float lr,
                        float* loss);
/* Data-parallel training (no reference counterpart): dcfr_mlp_backward
 * leaves this batch's gradients in the device buffer that
 * dcfr_mlp_gradients_device returns (flat padded layout, `count` floats;
 * the network's stream is synchronised on return). The caller sums that
 * buffer across ranks in place (an NCCL all-reduce) and synchronises, then
 * dcfr_mlp_adam_step applies one Adam step to the buffer times gscale (1 /
 * ranks for the mean). backward + adam_step(lr, 1) on one rank is
 * dcfr_mlp_train_step. */
int dcfr_mlp_backward(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t m, float* loss);
int dcfr_mlp_gradients_device(dcfr_mlp* n, float** grads, uint64_t* count);
int dcfr_mlp_adam_step(dcfr_mlp* n, float lr, float gscale);
/* The tensor-core GEMM itself: c = epi(a[m][k] x b[n][k]^T) with a, b bf16
 * (k contiguous), m and n multiples of 128, k of 64; epi 0: c f32; 1: c f32
 * + bias[n]; 2: z bf16 = acc + bias, c bf16 = gelu(z); 3: c bf16 = acc *
 * gelu'(z). ldc is the row stride of c (and z) in elements. */
int dcfr_gemm_bf16(const void* a, const void* b, void* c, int32_t m, int32_t n, int32_t k, int32_t epi,
                   const float* bias, void* z, int32_t ldc, void* stream);
/* The same GEMM launched `reps` times back to back on `stream` (no host
 * synchronisation between launches), timed with CUDA events on that stream:
 * *ms_per_launch is the mean device time of one launch. No reference
 * counterpart (the reference has no network). */
int dcfr_gemm_bf16_timed(const void* a, const void* b, void* c, int32_t m, int32_t n, int32_t k, int32_t epi,
                         const float* bias, void* z, int32_t ldc, int32_t reps, void* stream, float* ms_per_launch);

/* Largest hand count per side that dcfr_showdown_values_noalloc accepts. */
#define DCFR_NOALLOC_MAX_HANDS 1326

/* No counterpart in the reference: range-vs-range showdown values on one
 * river board, for callers that cannot allocate device memory (a host whose
 * device memory belongs to its own pool allocator, or a process held to a
 * fixed device-memory budget). It allocates nothing: its scratch is one
 * static device array of 192 KiB that every GPU loading the library holds
 * until exit. For each hero hand h,
 *   out[h] = win  * (sum of opp_reach over opponent hands weaker than h)
 *          + lose * (sum over stronger hands) + tie * (sum over equal hands),
 * counting only opponent hands that share no card with h (lose is signed:
 * pass a negative payoff). board (5 cards) and the two hand lists (2 card
 * ids per hand, no board cards, no repeats, at most DCFR_NOALLOC_MAX_HANDS
 * each) are host memory; opp_reach (n_opp floats) and out (n_hero floats)
 * are device memory; opp_reach entries must be finite and >= 0 (a call
 * given a negative, NaN or infinite entry writes NaN to every out entry).
 * stream is a cudaStream_t (NULL: the default stream) and the call is
 * asynchronous on it. Calls share the scratch array: calls whose work
 * overlaps on the GPU race and must be serialised by the caller. The first
 * call on each device does a one-time set-up with that device current and
 * caches it for the process (resetting the device while the library is
 * loaded is not supported); make that first call before any stream
 * capture. */
int dcfr_showdown_values_noalloc(const uint8_t board[5], const uint8_t* hero_cards, int32_t n_hero,
                                 const uint8_t* opp_cards, int32_t n_opp, const float* opp_reach, double win,
                                 double lose, double tie, float* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DCFR_H */
