// dcfr_showdown_values_noalloc: range-vs-range showdown values on one river
// board, computed by the fast-precision terminal kernels (terminal_fast.cu)
// with every scratch buffer in one file-scope static device array, so the
// call allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree. Examples are
// a host whose device memory is owned by its own pool allocator (a trainer
// sharing the GPU with a framework's caching allocator that has reserved
// the device), a process held to a fixed device-memory budget, and
// latency-sensitive loops where an allocation's implicit device
// synchronisation would stall other streams.
//
// Limits and sharing rules:
// - at most DCFR_NOALLOC_MAX_HANDS (1326) hands per side; larger sizes are
//   rejected with DCFR_ERR_INVALID_ARG;
// - the scratch array (192 KiB) lives in every device that loads the
//   library until the process exits;
// - all calls share the one array and it keeps the last call's contents;
//   every call rewrites all of it that must start from zero. Calls whose
//   work overlaps on the GPU (different streams, or different host threads
//   on one device) race on the array and give wrong results: serialise them;
// - the first call on each device does a one-time set-up with that device
//   current (resolving the array's device address and the terminal kernel's
//   shared-memory limit); make that first call before any stream capture.
//   The set-up is cached for the life of the process: resetting the device
//   (cudaDeviceReset) while the library is loaded is not supported;
// - opp_reach must be finite and >= 0 (reach probabilities times weights):
//   the exact fixed-point sums assume it. A call given a negative, NaN or
//   infinite entry writes NaN to every out entry instead of values.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/dcfr.h"
#include "engine.hpp"
#include "plan.hpp"

namespace dcfr {
void set_last_error(const std::string& msg);
}  // namespace dcfr

namespace {

using namespace dcfr;

constexpr int NA_MAX = DCFR_NOALLOC_MAX_HANDS;
constexpr int NA_HP = (NA_MAX + 7) & ~7;  // padded row length (1328)
constexpr int NA_CSTRIDE = 3 * NA_HP;     // scan elements per layout
constexpr int NA_LAYOUTS = 4;             // (board, fold) x (player 0, player 1)

// Layout of the scratch array. Player 0 is the hero (the traverser of the
// terminal kernel), player 1 the opponent.
struct Scratch {
  alignas(16) float reach[NA_HP];      // opponent reach, zero-padded
  alignas(16) float vals[NA_HP];       // hero values
  alignas(16) uint4 rec[NA_LAYOUTS][NA_HP];
  alignas(16) EntryD tables[2][NA_HP]; // strength-sorted hands per player
  alignas(16) uint32_t same[NA_HP];    // hero hand -> identical opponent hand
  alignas(16) uint16_t cat[NA_LAYOUTS][NA_CSTRIDE];
  alignas(16) uint16_t seg[NA_LAYOUTS][FAST_SEGS];
  alignas(16) FastTask task;
  alignas(16) uint8_t hc1[2][NA_HP];   // hand cards, padded with 255
  alignas(16) uint8_t hc2[2][NA_HP];
  alignas(16) uint8_t board[8];
  uint32_t count[2];
  uint32_t alive[2];
};

constexpr size_t SCRATCH_BYTES = 196608;  // 192 KiB
static_assert(sizeof(Scratch) <= SCRATCH_BYTES, "scratch layout exceeds the static array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

// Host-checked inputs, passed by value as the prep kernel's parameter
// (about 5.4 KB, within the 32 KB kernel-parameter limit).
struct PrepParams {
  uint8_t board[5];
  uint8_t cards[2][2 * NA_MAX];  // [player][2*hand + k]
  int n[2];
  double win, lose, tie;
};

// Fills everything the terminal kernels read: padded card arrays, the
// identical-hand map, the zero-padded reach row, the liveness flag and the
// single terminal task.
__global__ void __launch_bounds__(1024) noalloc_prep_kernel(Scratch* S, const __grid_constant__ PrepParams P,
                                                            const float* __restrict__ reach) {
  __shared__ uint16_t opp_of_combo[DCFR_NUM_COMBOS];
  const int tid = threadIdx.x;
  for (int i = tid; i < DCFR_NUM_COMBOS; i += blockDim.x) opp_of_combo[i] = 0xFFFF;
  if (tid < 8) S->board[tid] = tid < 5 ? P.board[tid] : 0;
  for (int q = 0; q < 2; q++)
    for (int h = tid; h < NA_HP; h += blockDim.x) {
      const bool in = h < P.n[q];
      S->hc1[q][h] = in ? P.cards[q][2 * h] : 255;
      S->hc2[q][h] = in ? P.cards[q][2 * h + 1] : 255;
    }
  // Entries that are negative, NaN or infinite: the call's output is NaN.
  int bad = 0;
  for (int h = tid; h < NA_HP; h += blockDim.x) {
    const float r = h < P.n[1] ? reach[h] : 0.0f;
    bad |= !(r >= 0.0f && r <= 3.402823466e38f);
    S->reach[h] = r;
  }
  bad = __syncthreads_or(bad);
  for (int j = tid; j < P.n[1]; j += blockDim.x) {
    const int a = P.cards[1][2 * j], b = P.cards[1][2 * j + 1];
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    opp_of_combo[hi * (hi - 1) / 2 + lo] = (uint16_t)j;
  }
  __syncthreads();
  for (int h = tid; h < NA_HP; h += blockDim.x) {
    uint32_t sm = NONE32;
    if (h < P.n[0]) {
      const int a = P.cards[0][2 * h], b = P.cards[0][2 * h + 1];
      const int hi = a > b ? a : b, lo = a > b ? b : a;
      const uint16_t j = opp_of_combo[hi * (hi - 1) / 2 + lo];
      sm = j == 0xFFFF ? NONE32 : (uint32_t)j;
    }
    S->same[h] = sm;
  }
  // A rejected row leaves the task dead (the terminal kernel skips it) and
  // the values NaN.
  if (bad)
    for (int h = tid; h < NA_HP; h += blockDim.x) S->vals[h] = __int_as_float(0x7fc00000);
  if (tid == 0) {
    S->alive[0] = bad ? 0 : 1;
    S->alive[1] = 0;
    FastTask t;
    t.kind = T_SHOWDOWN_BATCH;
    t.board = 0;
    t.slot = 0;
    t.row = 0;
    t.frow = NONE32;
    t.pad[0] = t.pad[1] = t.pad[2] = 0;
    t.a = P.win;
    t.b = P.lose;
    t.c = P.tie;
    t.d = 0.0;
    S->task = t;
  }
}

// Device address of a member of the scratch array (host code never
// dereferences the device pointer).
template <typename T>
T* member(Scratch* S, size_t offset) {
  return reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(S) + offset);
}
#define AT(T, field) member<T>(S, offsetof(Scratch, field))

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
Scratch* g_scratch_ptr[MAX_DEVICES] = {};

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

// Once per device, with that device current: the array's device address and
// the terminal kernel's dynamic shared-memory attribute.
int setup(Scratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(DCFR_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(DCFR_ERR_CUDA, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(DCFR_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    const int emax = fast_emax(NA_HP);
    if (fast_blocks_per_sm(NA_HP, emax, NA_CSTRIDE, NA_HP) <= 0)
      return fail(DCFR_ERR_CUDA, "terminal kernel does not fit this device's shared memory");
    g_scratch_ptr[dev] = static_cast<Scratch*>(p);
  }
  *out = g_scratch_ptr[dev];
  return DCFR_OK;
}

int check_hands(const uint8_t* cards, int n, uint64_t board_set, const char* who, PrepParams& P, int q) {
  if (n < 0 || n > NA_MAX)
    return fail(DCFR_ERR_INVALID_ARG, std::string(who) + ": hand count must be in 0..1326 (the scratch limit)");
  if (n > 0 && !cards) return fail(DCFR_ERR_INVALID_ARG, std::string(who) + ": cards is NULL");
  static thread_local uint8_t seen[DCFR_NUM_COMBOS];
  std::memset(seen, 0, sizeof seen);
  for (int h = 0; h < n; h++) {
    const int a = cards[2 * h], b = cards[2 * h + 1];
    if (a >= 52 || b >= 52 || a == b)
      return fail(DCFR_ERR_INVALID_ARG, std::string(who) + ": hand " + std::to_string(h) + " is not two distinct cards");
    if (((board_set >> a) & 1) || ((board_set >> b) & 1))
      return fail(DCFR_ERR_INVALID_ARG, std::string(who) + ": hand " + std::to_string(h) + " uses a board card");
    const int hi = a > b ? a : b, lo = a > b ? b : a;
    const int c = hi * (hi - 1) / 2 + lo;
    if (seen[c]) return fail(DCFR_ERR_INVALID_ARG, std::string(who) + ": hand " + std::to_string(h) + " is repeated");
    seen[c] = 1;
    P.cards[q][2 * h] = (uint8_t)a;
    P.cards[q][2 * h + 1] = (uint8_t)b;
  }
  P.n[q] = n;
  return DCFR_OK;
}

}  // namespace

extern "C" int dcfr_showdown_values_noalloc(const uint8_t board[5], const uint8_t* hero_cards, int32_t n_hero,
                                            const uint8_t* opp_cards, int32_t n_opp, const float* opp_reach,
                                            double win, double lose, double tie, float* out, void* stream) {
  if (!board) return fail(DCFR_ERR_INVALID_ARG, "board is NULL");
  static thread_local PrepParams P;
  std::memset(&P, 0, sizeof P);
  uint64_t board_set = 0;
  for (int k = 0; k < 5; k++) {
    if (board[k] >= 52 || ((board_set >> board[k]) & 1))
      return fail(DCFR_ERR_INVALID_BOARD, "board must be five distinct cards");
    board_set |= 1ull << board[k];
    P.board[k] = board[k];
  }
  int rc = check_hands(hero_cards, n_hero, board_set, "hero", P, 0);
  if (rc) return rc;
  if ((rc = check_hands(opp_cards, n_opp, board_set, "opponent", P, 1))) return rc;
  if (n_opp > 0 && !opp_reach) return fail(DCFR_ERR_INVALID_ARG, "opp_reach is NULL");
  if (n_hero > 0 && !out) return fail(DCFR_ERR_INVALID_ARG, "out is NULL");
  if (n_hero == 0) return DCFR_OK;
  P.win = win;
  P.lose = lose;
  P.tie = tie;

  Scratch* S = nullptr;
  if ((rc = setup(&S))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  uint8_t* hc1_0 = AT(uint8_t, hc1);
  uint8_t* hc1_1 = hc1_0 + NA_HP;
  uint8_t* hc2_0 = AT(uint8_t, hc2);
  uint8_t* hc2_1 = hc2_0 + NA_HP;
  EntryD* tables = AT(EntryD, tables);
  uint32_t* count = AT(uint32_t, count);
  uint16_t* cat = AT(uint16_t, cat);
  uint16_t* seg = AT(uint16_t, seg);
  uint4* rec = AT(uint4, rec);

  // Launch errors below are this call's: clear any left by earlier work on
  // this thread.
  (void)cudaGetLastError();
  noalloc_prep_kernel<<<1, 1024, 0, s>>>(S, P, opp_reach);
  launch_strength(AT(uint8_t, board), 1, hc1_0, hc2_0, hc1_1, hc2_1, n_hero, n_opp, tables, count, NA_HP, s);
  launch_fast_layouts(tables, count, NA_HP, 1, hc1_0, hc2_0, hc1_1, hc2_1, n_hero, n_opp, cat, seg, rec, NA_CSTRIDE,
                      s);
  FastArgs A;
  std::memset(&A, 0, sizeof A);
  A.reach = AT(float, reach);
  A.vals = AT(float, vals);
  A.alive = AT(uint32_t, alive);
  A.cat = cat;
  A.seg = seg;
  A.rec = rec;
  A.same = AT(uint32_t, same);
  A.cstride = NA_CSTRIDE;
  A.tstride = NA_HP;
  A.emax = fast_emax(NA_HP);
  A.n[0] = n_hero;
  A.n[1] = n_opp;
  A.hp[0] = (n_hero + 7) & ~7;
  A.hp[1] = (n_opp + 7) & ~7;
  A.stride = NA_HP;
  A.p = 0;
  launch_fast_terminal(A, AT(FastTask, task), 1, 1, s);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(DCFR_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  e = cudaMemcpyAsync(out, AT(float, vals), (size_t)n_hero * sizeof(float), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return fail(DCFR_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
  set_last_error("");
  return DCFR_OK;
}
