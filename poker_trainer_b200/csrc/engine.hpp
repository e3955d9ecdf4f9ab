// Device engine of libdcfr: owns the device copy of the game, the storage,
// the per-traversal plans and the captured CUDA graphs of one solver handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "game.hpp"
#include "plan.hpp"

struct dcfr_mlp;

namespace dcfr {

struct RowArgs;
struct TermArgs;

// Kernel launchers (kernels.cu).
void launch_down(int mode, int maxa, const RowArgs& A, const DownTask* tasks, int ntasks, int hp, cudaStream_t s);
void launch_up(int mode, int maxa, const RowArgs& A, const UpTask* tasks, int ntasks, int hp, cudaStream_t s);
void launch_fused_down(int mode, int maxa, const RowArgs& A, const FusedTree* trees, int ntrees,
                       const DownTask* tasks, int hp, cudaStream_t s);
void launch_fused_up(int mode, int maxa, const RowArgs& A, const FusedTree* trees, int ntrees, const UpTask* tasks,
                     int hp, cudaStream_t s);
void launch_terminal(const TermArgs& A, const TermGroup* groups, const TermLane* lanes, const TermTask* tasks,
                     int ntasks, cudaStream_t s);
cudaError_t terminal_kernel_setup();
size_t terminal_smem_bytes();
void launch_programs(const EntryD* tables, const uint32_t* count, int tstride, uint32_t* progs, uint32_t* prog_count,
                     uint32_t* posmap, int pstride, int nboards, cudaStream_t s);
void launch_hand_program(const uint8_t* c1, const uint8_t* c2, const uint32_t* same, int n, int npad,
                         uint32_t* fold_prog, uint2* emit_rec, cudaStream_t s);
void launch_strength(const uint8_t* boards, int nboards, const uint8_t* hc1_0, const uint8_t* hc2_0,
                     const uint8_t* hc1_1, const uint8_t* hc2_1, int n0, int n1, EntryD* out, uint32_t* count,
                     int tstride, cudaStream_t s);
void launch_fast_layouts(const EntryD* tables, const uint32_t* count, int tstride, int nboards, const uint8_t* hc1_0,
                         const uint8_t* hc2_0, const uint8_t* hc1_1, const uint8_t* hc2_1, int n0, int n1,
                         uint16_t* cat, uint16_t* seg, uint4* rec, int cstride, cudaStream_t s);
void launch_fast_terminal(const FastArgs& A, const FastTask* tasks, int ntasks, int max_blocks, cudaStream_t s);
void launch_fast_terminal64(const FastArgs64& A, const FastTask* tasks, int ntasks, int max_blocks, cudaStream_t s);
void launch_warp_terminal(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                          int warps,
                          int max_blocks, cudaStream_t s);
void launch_warp_terminal64(const FastArgs64& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                            int warps,
                            int max_blocks, cudaStream_t s);
int warp_terminal_setup(int stride, int cstride, int tstride, int rsize, int max_warps, int& blocks_per_sm);
int group_terminal_setup(int stride, int cstride, int tstride, int& blocks_per_sm);
void launch_group_terminal(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                           int groups, int max_blocks, cudaStream_t s);
int panel_terminal_setup(int hpo, int hpp, int cstride, int tstride, int T, int& blocks_per_sm);
int warp_terminal_dyn_setup(int stride, int cstride, int tstride, int max_warps, int& blocks_per_sm);
void launch_fast_terminal_dyn(const FastArgs& A, const FastTask* tasks, int ntasks, int max_blocks, uint32_t* counter,
                              cudaStream_t s);
void launch_warp_terminal_dyn(const FastArgs& A, const FastTask* tasks, const TermUnit* units, int nunits, int ntasks,
                              int warps, int max_blocks, uint32_t* counter, cudaStream_t s);
void launch_panel_terminal(const FastArgs& A, const FastTask* tasks, const PanelD* panels, int npanels, int T, int e,
                           int max_blocks, cudaStream_t s);
// FP64 best-response oracle kernels (br64.cu).
void launch_down64(const Row64Args& A, const DownTask* tasks, int ntasks, int hp, cudaStream_t s);
void launch_up64(int mode, const Row64Args& A, const UpTask* tasks, int ntasks, int hp, cudaStream_t s);
void launch_fused_down64(const Row64Args& A, const FusedTree* trees, int ntrees, const DownTask* tasks, cudaStream_t s);
void launch_fused_up64(int mode, const Row64Args& A, const FusedTree* trees, int ntrees, const UpTask* tasks,
                       cudaStream_t s);
int fast_emax(int tstride);
int fast_blocks_per_sm(int stride, int emax, int cstride, int tstride);
void launch_evaluate(const unsigned long long* masks, uint32_t* out, int n, cudaStream_t s);
void launch_five_card_counts(unsigned long long* counts, cudaStream_t s);
// counter non-null: also advance the DCFR iteration (t += 1, the discounts
// of iteration t from the table into cur).
void launch_traversal_start(uint32_t* alive, int nslots, float* reach, const float* root_row, int stride,
                            uint32_t* counter, const DiscountD* table, uint32_t table_len, DiscountD* cur,
                            cudaStream_t s);
// Storage blocks between the device layout and the reference's packed
// layout; elem_bytes 4 (f32) or 2 (compressed storage).
void launch_storage_pack(int elem_bytes, const void* dev, void* packed, const StorageBlockD* blocks, int nblocks,
                         cudaStream_t s);
void launch_storage_unpack(int elem_bytes, void* dev, const void* packed, const StorageBlockD* blocks, int nblocks,
                           cudaStream_t s);

// Status of a failed call: code + message.
struct Status {
  int code = DCFR_OK;
  std::string msg;
  bool ok() const { return code == DCFR_OK; }
};

// One traversal plan: traverser p over the subtree at `root`.
struct Plan {
  int p = 0;
  uint32_t root = 0;
  uint32_t nslots = 0;
  // A level's tasks, sorted by kind: count[k] tasks of kind k from first on.
  struct Level {
    uint32_t first = 0, count = 0;
    int maxa = 0;
    uint32_t kind_count[3] = {0, 0, 0};
  };
  std::vector<Level> down, up;  // chance nodes by layer (down[l]: splits; up[l]: sums)
  std::vector<std::vector<Level>> seg_down, seg_up;  // wide segments: [layer][depth]
  std::vector<DownTask> h_down;
  std::vector<UpTask> h_up;
  std::vector<TermGroup> h_groups;
  std::vector<TermLane> h_lanes;
  std::vector<TermTask> h_tasks;
  std::vector<FastTask> h_fast;  // fast precision: one task per terminal
  std::vector<TermUnit> h_units; // runs of h_fast on one layout (warp terminal kernel)
  TermUnit* d_units = nullptr;
  std::vector<PanelD> h_panels;  // panels of h_fast (panel terminal kernel)
  PanelD* d_panels = nullptr;
  std::vector<LeafTask> h_leaves; // depth-limited solves: the leaves of this traversal
  LeafTask* d_leaves = nullptr;
  // Fused river subtrees (one block each) and their tasks.
  std::vector<FusedTree> h_trees;
  std::vector<DownTask> h_fdown;
  std::vector<UpTask> h_fup;
  int fused_maxa = 0;
  // Segments by layer (the number of chance nodes above): [first tree, count].
  std::vector<std::pair<uint32_t, uint32_t>> tree_layers;
  FusedTree* d_trees = nullptr;
  DownTask* d_fdown = nullptr;
  UpTask* d_fup = nullptr;
  struct Wave {
    uint32_t first = 0, count = 0, groups = 0;
  };
  std::vector<Wave> waves;
  TermTask* d_tasks = nullptr;
  DownTask* d_down = nullptr;
  UpTask* d_up = nullptr;
  TermGroup* d_groups = nullptr;
  TermLane* d_lanes = nullptr;
  FastTask* d_fast = nullptr;
  int kernels = 0;  // kernel launches per traversal
  int class_kernels[DCFR_KERNEL_CLASSES] = {0, 0, 0, 0};
  double class_bytes[DCFR_KERNEL_CLASSES] = {0, 0, 0, 0};  // compulsory bytes per traversal (CFR mode)
  uint64_t nodes = 0;
  ~Plan();
};

// Leaf evaluation of depth-limited solves (leaf.cu).
struct LeafArgs {
  const float* reach;       // reach rows (slots x stride)
  float* vals;              // value rows (nodes x stride)
  const uint32_t* alive;
  float* leaf_reach[2];     // per player: its reach at each leaf [leaves][stride], hand order
  const uint16_t* combos[2];// per player: combo id of each hand
  float* x;                 // network input [leaves * nc][in_dim]
  const float* y;           // network output, row stride ldy: EV / pot per combo, player 0 then 1
  int ldy;
  const uint8_t* cards;     // the nc cards dealt at the leaves (ascending)
  int nc;
  int board[3];
  int n[2];
  int stride;
  int p;
  float factor;             // chance factor of the leaf's deal (tree.rs:520-542)
  double norm;              // 1 / num_combinations
};
void launch_leaf_capture(const LeafArgs& A, const LeafTask* tasks, int ntasks, cudaStream_t s);
void launch_leaf_inputs(const LeafArgs& A, const LeafTask* tasks, int ntasks, const uint8_t* hc1_0,
                        const uint8_t* hc2_0, const uint8_t* hc1_1, const uint8_t* hc2_1, cudaStream_t s);
void launch_leaf_values(const LeafArgs& A, const LeafTask* tasks, int ntasks, const uint8_t* hc1_p,
                        const uint8_t* hc2_p, const uint8_t* hc1_o, const uint8_t* hc2_o, int hp, cudaStream_t s);
// The leaf-value network (mlp.cu): shape check, and a forward pass enqueued on
// stream s (no synchronisation) whose padded output y has row stride ldy.
int mlp_shape(const dcfr_mlp* n, int* in_dim, int* out_dim, int* max_batch);
int mlp_enqueue_forward(dcfr_mlp* n, const float* x, int m, cudaStream_t s, const float** y, int* ldy);

class Engine {
 public:
  static Status create(const dcfr_config& cfg, std::unique_ptr<Engine>& out);
  // A depth-limited solve: the tree ends at the deal of leaf_street, whose
  // nodes are valued by `net` (not owned; must outlive the solver).
  static Status create_depth_limited(const dcfr_config& cfg, dcfr_mlp* net, int leaf_street,
                                     std::unique_ptr<Engine>& out);
  ~Engine();

  Game g;
  uint32_t iterations = 0;
  double last_exploitability;
  uint64_t launches = 0;
  double last_iterate_ms = 0.0;
  double last_solve_ms = 0.0;
  dcfr_setup_profile setup{};

  Status iterate(uint32_t n);
  Status iterate_profiled(uint32_t n, dcfr_kernel_profile& out);
  Status sync();
  Status exploitability(double& out);
  // The same exploitability with every reach and value row in double
  // (br64.cu): the FP64 best-response oracle of a solve.
  Status exploitability_fp64(double& out, double br[2]);
  Status root_values(double out[2]);
  Status traverse(int p, int mode, uint32_t t, float* out);
  Status solve(const dcfr_solve_options& opts, const volatile int32_t* cancel, dcfr_progress_cb cb, void* user,
               dcfr_progress& out);
  Status download(float* regrets, float* sums);
  Status upload(const float* regrets, const float* sums);
  // 16-bit compressed storage in the reference layout (storage.rs:92-97):
  // len values of each kind, one scale of each kind per decision node slot.
  bool compressed() const { return compressed_; }
  uint64_t slots() const { return g.player_nodes; }
  Status download_compressed(int16_t* regrets, uint16_t* sums, float* rscale, float* sscale);
  Status upload_compressed(const int16_t* regrets, const uint16_t* sums, const float* rscale, const float* sscale);
  Status set_iterations(uint32_t t);
  Status query(const std::vector<dcfr_step>& path, dcfr_node_info& info, std::vector<Act>& actions,
               std::vector<uint16_t>& combos, std::vector<float>& strategy, std::vector<float>& ev,
               std::vector<float>& reach);
  Status ranges_after(const std::vector<dcfr_step>& path, float out[2][DCFR_NUM_COMBOS]);
  Status actions_at(const std::vector<dcfr_step>& path, std::vector<Act>& out, bool& decision);
  double iteration_bytes() const;
  // The f32 traversals' terminal kernel (DCFR_TERMINAL_*) and panel width.
  void terminal_kernel(int32_t& kernel, int32_t& per_panel) const {
    kernel = !fast_ ? DCFR_TERMINAL_EXACT : term_group_ ? DCFR_TERMINAL_GROUP : term_kernel_;
    per_panel = fast_ && term_kernel_ == TK_PANEL ? panel_T_ : 0;
  }
  int isomorphic_pairs() const;
  // Offset of a decision node's block in the reference storage layout.
  Status node_storage(const std::vector<dcfr_step>& path, uint64_t& offset, int& num_actions, int& num_hands);
  bool depth_limited() const { return net_ != nullptr; }
  // Overwrites a decision node's blocks (reference layout [actions][hands]).
  Status write_node(const std::vector<dcfr_step>& path, const float* regrets, const float* sums);

 private:
  cudaStream_t stream_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  int hp_[2] = {0, 0};
  int stride_ = 0;
  std::vector<uint64_t> gpu_off_;  // per node: float offset of a player node's block
  uint64_t gpu_len_ = 0;
  // Device buffers.
  float* regrets_ = nullptr;
  float* sums_ = nullptr;
  bool compressed_ = false;
  int16_t* rq_ = nullptr;   // compressed storage (GPU layout) and per-slot scales
  uint16_t* sq_ = nullptr;
  float* rscale_ = nullptr;
  float* sscale_ = nullptr;
  Status download_compressed_raw(std::vector<int16_t>& rq, std::vector<uint16_t>& sq, std::vector<float>& rs,
                                 std::vector<float>& ss);
  // Transfers between the device storage and the reference layout, through
  // a device staging buffer in chunks of whole decision nodes.
  struct StorageChunk {
    uint32_t first, count;  // blocks sblk_[first, first + count)
    uint64_t host, len;     // elements [host, host + len) of the reference layout
  };
  std::vector<StorageChunk> schunks_;
  StorageBlockD* sblk_ = nullptr;
  uint64_t stage_len_ = 0;  // elements of the staging buffer (the largest chunk)
  Status storage_chunks();
  Status storage_out(const void* dev, void* host, int elem_bytes);
  Status storage_in(void* dev, const void* host, int elem_bytes);
  float* reach_ = nullptr;
  float* vals_ = nullptr;
  uint32_t* alive_ = nullptr;
  float* root_rows_ = nullptr;   // [2][stride] opponent root weights per traverser
  float* root_out_ = nullptr;    // [2][stride] root values after a traversal pair
  uint8_t* hc1_[2] = {nullptr, nullptr};
  uint8_t* hc2_[2] = {nullptr, nullptr};
  uint32_t* same_[2] = {nullptr, nullptr};
  uint16_t* perm_ = nullptr;
  uint8_t* chance_cards_ = nullptr;
  IsoRefD* iso_ = nullptr;
  EntryD* tables_ = nullptr;
  uint32_t* table_count_ = nullptr;
  int tstride_ = 0;
  uint32_t* progs_ = nullptr;
  uint32_t* prog_count_ = nullptr;
  uint32_t* posmap_ = nullptr;
  uint32_t* fold_prog_[2] = {nullptr, nullptr};
  uint2* emit_rec_[2] = {nullptr, nullptr};
  int pstride_ = 0;
  float* warp_scratch_ = nullptr;
  size_t warp_scratch_floats_ = 0;
  double* group_scratch_ = nullptr;
  uint32_t* counters_ = nullptr;
  int wave_tasks_ = 0, wave_groups_ = 0;
  // Fast precision (terminal_fast.cu): scan layouts per (layout, traverser).
  bool fast_ = true;
  uint16_t* fcat_ = nullptr;
  uint16_t* fseg_ = nullptr;
  uint4* frec_ = nullptr;
  int fcstride_ = 0, femax_ = 0, fast_blocks_ = 0;
  // Warp terminal kernel: warps per block and blocks (float rows, double rows).
  int term_warps_[2] = {0, 0}, term_blocks_[2] = {0, 0};
  // Terminal kernel of the f32 solve in fast precision, and the panel
  // kernel's terminals per panel, elements per thread and blocks.
  enum TermKernel { TK_PANEL = DCFR_TERMINAL_PANEL, TK_WARP = DCFR_TERMINAL_WARP, TK_BLOCK = DCFR_TERMINAL_BLOCK };
  int term_kernel_ = TK_PANEL;
  int panel_T_ = 0, panel_E_ = 0, panel_blocks_ = 0;
  // The warp kernel's scheduling: static task ranges per block, or chunks
  // claimed from term_counter_ (dynamic).
  bool term_dynamic_ = false;
  int dyn_warps_ = 0, dyn_blocks_ = 0;
  // Short rows: two warps per terminal (terminal_group.cu) instead of one.
  bool term_group_ = false, term_group_auto_ = false;
  int group_groups_ = 0, group_blocks_ = 0, term_sms_ = 0;
  uint32_t* term_counter_ = nullptr;
  // Depth-limited solves: the leaf-value network and its buffers.
  dcfr_mlp* net_ = nullptr;
  float* leaf_reach_[2] = {nullptr, nullptr};
  float* leaf_x_ = nullptr;
  uint8_t* leaf_cards_ = nullptr;
  uint16_t* combos_[2] = {nullptr, nullptr};
  int leaf_nc_ = 0;
  float leaf_factor_ = 0.0f;
  Status init_leaves();
  void enqueue_leaves(const Plan& plan);
  Status leaf_status_;
  // FP64 best-response rows, allocated on first use.
  double* reach64_ = nullptr;
  double* vals64_ = nullptr;
  double* root_rows64_ = nullptr;
  Status ensure_fast_layouts();
  Status fp64_root_values(int mode, double out[2]);
  DiscountD* disc_table_ = nullptr;
  uint32_t disc_len_ = 0;
  DiscountD* cur_disc_ = nullptr;
  uint32_t* counter_ = nullptr;
  uint64_t max_slots_ = 0;
  std::vector<uint32_t> cc_off_, iso_first_;
  std::unique_ptr<Plan> full_[2];
  cudaGraphExec_t iter_graph_ = nullptr, br_graph_ = nullptr, avg_graph_ = nullptr;
  // Profiled iteration graph: event-record nodes at kernel-class boundaries.
  struct Mark {
    cudaGraphNode_t node;
    int cls;  // class of the interval that ends at this event (-1: first)
  };
  std::vector<Mark>* marking_ = nullptr;  // set while capturing the profiled graph
  cudaGraph_t prof_graph_ = nullptr;
  cudaGraphExec_t prof_exec_ = nullptr;
  std::vector<Mark> marks_;
  std::vector<cudaEvent_t> prof_events_;
  Status mark_status_;
  void mark(int cls);
  Status capture_profiled_graph();
  int iter_kernels_ = 0, pair_kernels_ = 0;

  Status init();
  Status alloc_storage();
  Status build_plan(uint32_t root, int p, Plan& plan);
  Status upload_plan(Plan& plan);
  void row_args(int p, RowArgs& A) const;
  void term_args(int p, TermArgs& A) const;
  void fast_args(int p, FastArgs& A) const;
  void enqueue_traversal(const Plan& plan, int mode, const float* root_row, float* root_out, bool advance = false);
  Status ensure_discounts(uint32_t max_t);
  Status capture_graphs();
  Status capture_eval_graphs();
  Status solve_loop(const dcfr_solve_options& opts, const volatile int32_t* cancel, dcfr_progress_cb cb, void* user,
                    dcfr_progress& progress);
  void free_graphs();
  Status mode_root_values(int mode, double out[2]);
  Status walk(const std::vector<dcfr_step>& path, uint32_t& node, std::vector<float> reach[2],
              std::vector<uint32_t> to_canon[2]);
  Status avg_strategy(uint32_t node, std::vector<float>& s);
  Status subtree_values(uint32_t root, int p, const std::vector<float>& opp_reach, std::vector<float>& out);
  Status root_child_values(int q, const std::vector<float>& opp_reach, std::vector<std::vector<float>>& child);
};

Status cuda_status(cudaError_t e, const char* what);

}  // namespace dcfr
