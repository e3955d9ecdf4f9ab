// The leaf-value network: an MLP trained and evaluated on the GPU with the
// project's own BF16 tcgen05 GEMM (gemm_tc.cuh), FP32 accumulation and FP32
// master weights. No counterpart in the reference solver.
//
// Shapes: input in_dim -> `layers` hidden layers of width `hidden` with GELU
// -> linear output out_dim. Every dimension is padded to a multiple of 128
// (the GEMM tile); padded inputs, weights and outputs are zero and carry no
// gradient. Weights live in FP32 (Adam master copy, layout W_t[out][in]) and
// in two BF16 copies: W_t[out][in] (B operand of the forward GEMM) and
// W[in][out] (B operand of the input-gradient GEMM).
//
// Forward: X_{l+1} = gelu(X_l W_l + b_l) (pre-activation Z_l kept in BF16),
// Y = X_L W_L + b_L in FP32.
// Loss: sum over valid outputs of mask * (Y - T)^2 / sum(mask).
// Backward: dW_t[l] = dY_l^T X_l and db_l = column sums of dY_l (FP32);
// dY_{l-1} = (dY_l W_l) * gelu'(Z_{l-1}) fused in the GEMM epilogue.
// Adam updates the FP32 weights, which are then copied to the BF16 layouts.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/dcfr.h"
#include "engine.hpp"
#include "gemm_tc.cuh"

namespace dcfr {
void set_last_error(const std::string& msg);
}

namespace {

using namespace dcfr;
using bf16 = __nv_bfloat16;

int fail(int code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

#define MK(call)                                                                       \
  do {                                                                                 \
    cudaError_t _e = (call);                                                           \
    if (_e != cudaSuccess) return fail(DCFR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
  } while (0)

inline int pad128(int x) { return (x + 127) / 128 * 128; }

// cuTensorMapEncodeTiled through the runtime's driver entry point.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of a row-major bf16 matrix [rows][cols] (cols contiguous), read
// in 128-row x 64-column boxes with the 128-byte swizzle.
int make_map(CUtensorMap* map, const void* base, uint64_t rows, uint64_t cols) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(DCFR_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
  if (((uintptr_t)base & 15) || (cols * 2) % 16) return fail(DCFR_ERR_INVALID_ARG, "GEMM operand is not 16-byte aligned");
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {GEMM_BK, GEMM_BM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(DCFR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return DCFR_OK;
}

// C = epi(A[M][K] x B[N][K]^T); M, N multiples of 128, K of 64.
int gemm(const bf16* A, const bf16* B, int M, int N, int K, int epi, void* C, int ldc, bf16* z, const float* bias,
         int* err, cudaStream_t s) {
  if (M % GEMM_BM || N % GEMM_BN || K % GEMM_BK || M <= 0 || N <= 0 || K <= 0)
    return fail(DCFR_ERR_INVALID_ARG, "GEMM: M and N must be multiples of 128 and K of 64");
  static bool attr = false;
  if (!attr) {
    MK(cudaFuncSetAttribute(gemm_bf16_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
    attr = true;
  }
  CUtensorMap ma, mb;
  int rc = make_map(&ma, A, (uint64_t)M, (uint64_t)K);
  if (rc) return rc;
  if ((rc = make_map(&mb, B, (uint64_t)N, (uint64_t)K))) return rc;
  GemmArgs G{C, z, bias, ldc, epi, M, N, K, err};
  gemm_bf16_tc_kernel<<<dim3((unsigned)(N / GEMM_BN), (unsigned)(M / GEMM_BM)), GEMM_THREADS, GEMM_SMEM, s>>>(ma, mb, G);
  MK(cudaGetLastError());
  return DCFR_OK;
}

// out[c][r] = in[r][c] (bf16), tiles of 32 x 32 through shared memory.
__global__ void transpose_bf16(const bf16* __restrict__ in, bf16* __restrict__ out, int rows, int cols) {
  __shared__ bf16 t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : __float2bfloat16(0.0f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)c * rows + r] = t[threadIdx.x][i];
  }
}

void transpose(const bf16* in, bf16* out, int rows, int cols, cudaStream_t s) {
  transpose_bf16<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, s>>>(in, out, rows, cols);
}

// Row-major f32 [rows][cols] into a zero-padded bf16 [prow][pcol].
__global__ void pack_bf16(const float* __restrict__ in, int rows, int cols, bf16* __restrict__ out, int prow, int pcol) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)prow * pcol) return;
  const int r = (int)(i / pcol), c = (int)(i % pcol);
  out[i] = __float2bfloat16(r < rows && c < cols ? in[(size_t)r * cols + c] : 0.0f);
}

// f32 -> bf16, same layout; and f32 W_t[n][k] -> bf16 W[k][n].
__global__ void f32_to_bf16(const float* __restrict__ in, bf16* __restrict__ out, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16(in[i]);
}

__global__ void f32_transpose_bf16(const float* __restrict__ in, bf16* __restrict__ out, int rows, int cols) {
  __shared__ float t[32][33];
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < rows && c < cols) ? in[(size_t)r * cols + c] : 0.0f;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += 8) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[(size_t)c * rows + r] = __float2bfloat16(t[threadIdx.x][i]);
  }
}

// count[0] = number of valid outputs (sum of the mask, or rows * cols).
__global__ void mask_count(const float* __restrict__ mask, size_t n, float* __restrict__ count) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float c = i < n ? (mask ? mask[i] : 1.0f) : 0.0f;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c != 0.0f) atomicAdd(count, c);
}

// dY = 2 * mask * (Y - T) / count (bf16) and loss += mask * (Y - T)^2 / count,
// over the padded [prow][pcol] output; T and mask are [rows][cols] f32.
__global__ void loss_grad(const float* __restrict__ Y, const float* __restrict__ T, const float* __restrict__ mask,
                          int rows, int cols, int prow, int pcol, const float* __restrict__ count,
                          bf16* __restrict__ dY, float* __restrict__ loss) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float inv_count = *count > 0.0f ? 1.0f / *count : 0.0f;
  float l = 0.0f;
  if (i < (size_t)prow * pcol) {
    const int r = (int)(i / pcol), c = (int)(i % pcol);
    float g = 0.0f;
    if (r < rows && c < cols) {
      const size_t j = (size_t)r * cols + c;
      const float m = mask ? mask[j] : 1.0f;
      const float d = Y[i] - T[j];
      g = 2.0f * m * d * inv_count;
      l = m * d * d * inv_count;
    }
    dY[i] = __float2bfloat16(g);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0f) atomicAdd(loss, l);
}

// db[c] = sum over rows of dY[r][c].
__global__ void column_sums(const bf16* __restrict__ dY, int rows, int cols, float* __restrict__ db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float acc = 0.0f;
  for (int r = 0; r < rows; r++) acc += __bfloat162float(dY[(size_t)r * cols + c]);
  db[c] = acc;
}

// Adam on the f32 master copy; gradients of padded entries are zero by
// construction (pmask marks the real entries).
__global__ void adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                     const uint8_t* __restrict__ pmask, size_t n, float lr, float b1, float b2, float eps, float c1,
                     float c2, float gscale) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !pmask[i]) return;
  const float gi = g[i] * gscale;
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void copy_rows_f32(const float* __restrict__ in, int pcol, int rows, int cols, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (size_t)rows * cols) out[i] = in[(i / cols) * pcol + (i % cols)];
}

inline unsigned blocks_for(size_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

struct dcfr_mlp {
  int in_dim, out_dim, hidden, layers;  // `layers` hidden layers + 1 output layer
  int max_batch;
  std::vector<int> kin, nout;           // padded dims per layer (L + 1 layers)
  std::vector<size_t> woff, boff;       // offsets of W_t and b in the flat parameter arrays
  size_t nparams = 0, nw = 0;
  float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // flat: all W_t then all b
  uint8_t* pmask = nullptr;
  std::vector<bf16*> wt_bf, w_bf;       // per layer: [N][K] and [K][N]
  std::vector<bf16*> X, Z;              // activations [Mp][kin[l]] (X_0 = input) and pre-activations
  std::vector<bf16*> dY;                // [Mp][nout[l]]
  bf16 *tA = nullptr, *tB = nullptr;    // transposes for the weight-gradient GEMM
  float* Y = nullptr;                   // [Mp][nout[L]]
  float* loss = nullptr;
  int* err = nullptr;
  int step = 0;
  cudaStream_t stream = nullptr;
  ~dcfr_mlp() {
    for (void* p : std::vector<void*>{w, g, m, v, pmask, tA, tB, Y, loss, err}) cudaFree(p);
    for (auto* p : wt_bf) cudaFree(p);
    for (auto* p : w_bf) cudaFree(p);
    for (auto* p : X) cudaFree(p);
    for (auto* p : Z) cudaFree(p);
    for (auto* p : dY) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

int refresh_bf16(dcfr_mlp* n) {
  const int L = n->layers + 1;
  for (int l = 0; l < L; l++) {
    const size_t cnt = (size_t)n->nout[l] * n->kin[l];
    f32_to_bf16<<<blocks_for(cnt, 256), 256, 0, n->stream>>>(n->w + n->woff[l], n->wt_bf[l], cnt);
    f32_transpose_bf16<<<dim3((n->kin[l] + 31) / 32, (n->nout[l] + 31) / 32), dim3(32, 8), 0, n->stream>>>(
        n->w + n->woff[l], n->w_bf[l], n->nout[l], n->kin[l]);
  }
  MK(cudaGetLastError());
  return DCFR_OK;
}

int forward(dcfr_mlp* n, const float* x, int M, int Mp, cudaStream_t s) {
  int rc;
  pack_bf16<<<blocks_for((size_t)Mp * n->kin[0], 256), 256, 0, s>>>(x, M, n->in_dim, n->X[0], Mp, n->kin[0]);
  for (int l = 0; l < n->layers; l++)
    if ((rc = gemm(n->X[l], n->wt_bf[l], Mp, n->nout[l], n->kin[l], EPI_BIAS_GELU, n->X[l + 1], n->nout[l], n->Z[l],
                   n->w + n->boff[l], n->err, s)))
      return rc;
  const int L = n->layers;
  return gemm(n->X[L], n->wt_bf[L], Mp, n->nout[L], n->kin[L], EPI_BIAS_F32, n->Y, n->nout[L], nullptr,
              n->w + n->boff[L], n->err, s);
}

int forward(dcfr_mlp* n, const float* x, int M, int Mp) { return forward(n, x, M, Mp, n->stream); }

// Gradients of the loss into n->g (and the loss into n->loss).
int backward(dcfr_mlp* n, const float* target, const float* mask, int M, int Mp) {
  const int L = n->layers;
  // loss[0]: the loss; loss[1]: the number of valid outputs (the normaliser).
  MK(cudaMemsetAsync(n->loss, 0, 8, n->stream));
  MK(cudaMemsetAsync(n->g, 0, n->nparams * 4, n->stream));
  const size_t nt = (size_t)M * n->out_dim;
  mask_count<<<blocks_for(nt, 256), 256, 0, n->stream>>>(mask, nt, n->loss + 1);
  loss_grad<<<blocks_for((size_t)Mp * n->nout[L], 256), 256, 0, n->stream>>>(
      n->Y, target, mask, M, n->out_dim, Mp, n->nout[L], n->loss + 1, n->dY[L], n->loss);
  int rc;
  for (int l = L; l >= 0; l--) {
    const int K = n->kin[l], N = n->nout[l];
    // dW_t[l] [N][K] = dY_l^T X_l: operands dY_l^T [N][Mp] and X_l^T [K][Mp].
    transpose(n->dY[l], n->tA, Mp, N, n->stream);
    transpose(n->X[l], n->tB, Mp, K, n->stream);
    if ((rc = gemm(n->tA, n->tB, N, K, Mp, EPI_F32, n->g + n->woff[l], K, nullptr, nullptr, n->err, n->stream)))
      return rc;
    column_sums<<<blocks_for(N, 128), 128, 0, n->stream>>>(n->dY[l], Mp, N, n->g + n->boff[l]);
    if (l > 0) {
      // dY_{l-1} = (dY_l W_l) * gelu'(Z_{l-1}): B operand W_l as [K][N].
      if ((rc = gemm(n->dY[l], n->w_bf[l], Mp, K, N, EPI_GELU_GRAD, n->dY[l - 1], K, n->Z[l - 1], nullptr, n->err,
                     n->stream)))
        return rc;
    }
  }
  MK(cudaGetLastError());
  return DCFR_OK;
}

int check_err(dcfr_mlp* n) {
  int e = 0;
  MK(cudaMemcpyAsync(&e, n->err, 4, cudaMemcpyDeviceToHost, n->stream));
  MK(cudaStreamSynchronize(n->stream));
  if (e) return fail(DCFR_ERR_DEVICE_TIMEOUT, "tensor-core GEMM: a bounded wait gave up (code " + std::to_string(e) + ")");
  return DCFR_OK;
}

int batch_ok(dcfr_mlp* n, int M) {
  if (M <= 0 || M > n->max_batch) return fail(DCFR_ERR_INVALID_ARG, "batch size out of range");
  return DCFR_OK;
}

}  // namespace

namespace dcfr {

int mlp_shape(const dcfr_mlp* n, int* in_dim, int* out_dim, int* max_batch) {
  if (!n) return fail(DCFR_ERR_INVALID_ARG, "NULL network");
  *in_dim = n->in_dim;
  *out_dim = n->out_dim;
  *max_batch = n->max_batch;
  return DCFR_OK;
}

// The network's forward pass on stream s, nothing synchronised: a solver
// enqueues it between its kernels (and captures it in its graphs). y is the
// network's own padded output buffer, valid until its next forward pass.
int mlp_enqueue_forward(dcfr_mlp* n, const float* x, int m, cudaStream_t s, const float** y, int* ldy) {
  int rc = batch_ok(n, m);
  if (rc) return rc;
  if ((rc = forward(n, x, m, pad128(m), s))) return rc;
  *y = n->Y;
  *ldy = n->nout[n->layers];
  return DCFR_OK;
}

}  // namespace dcfr

extern "C" {

int dcfr_gemm_bf16(const void* a, const void* b, void* c, int32_t m, int32_t n, int32_t k, int32_t epi,
                   const float* bias, void* z, int32_t ldc, void* stream) {
  int* err = nullptr;
  MK(cudaMalloc(&err, 4));
  MK(cudaMemset(err, 0, 4));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = gemm(static_cast<const bf16*>(a), static_cast<const bf16*>(b), m, n, k, epi, c, ldc, static_cast<bf16*>(z),
                bias, err, s);
  int e = 0;
  if (!rc) {
    MK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, s));
    MK(cudaStreamSynchronize(s));
  }
  cudaFree(err);
  if (rc) return rc;
  if (e) return fail(DCFR_ERR_DEVICE_TIMEOUT, "tensor-core GEMM: a bounded wait gave up");
  set_last_error("");
  return DCFR_OK;
}

int dcfr_gemm_bf16_timed(const void* a, const void* b, void* c, int32_t m, int32_t n, int32_t k, int32_t epi,
                         const float* bias, void* z, int32_t ldc, int32_t reps, void* stream, float* ms_per_launch) {
  if (reps <= 0 || !ms_per_launch) return fail(DCFR_ERR_INVALID_ARG, "reps must be positive; ms_per_launch not NULL");
  int* err = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  MK(cudaMalloc(&err, 4));
  MK(cudaMemset(err, 0, 4));
  MK(cudaEventCreate(&e0));
  MK(cudaEventCreate(&e1));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = 0, e = 0;
  MK(cudaEventRecord(e0, s));
  for (int r = 0; r < reps && !rc; r++)
    rc = gemm(static_cast<const bf16*>(a), static_cast<const bf16*>(b), m, n, k, epi, c, ldc, static_cast<bf16*>(z),
              bias, err, s);
  MK(cudaEventRecord(e1, s));
  if (!rc) {
    MK(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, s));
    MK(cudaStreamSynchronize(s));
    float ms = 0.0f;
    MK(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_launch = ms / (float)reps;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(err);
  if (rc) return rc;
  if (e) return fail(DCFR_ERR_DEVICE_TIMEOUT, "tensor-core GEMM: a bounded wait gave up");
  set_last_error("");
  return DCFR_OK;
}

int dcfr_mlp_create(int32_t in_dim, int32_t hidden, int32_t layers, int32_t out_dim, int32_t max_batch,
                    uint64_t seed, dcfr_mlp** out) {
  if (!out || in_dim <= 0 || out_dim <= 0 || hidden <= 0 || hidden % 128 || layers < 1 || max_batch <= 0)
    return fail(DCFR_ERR_INVALID_ARG, "MLP shape: positive dims, hidden a multiple of 128, at least one layer");
  std::unique_ptr<dcfr_mlp> n(new dcfr_mlp());
  n->in_dim = in_dim;
  n->out_dim = out_dim;
  n->hidden = hidden;
  n->layers = layers;
  n->max_batch = max_batch;
  const int L = layers + 1;
  for (int l = 0; l < L; l++) {
    n->kin.push_back(l == 0 ? pad128(in_dim) : hidden);
    n->nout.push_back(l == layers ? pad128(out_dim) : hidden);
  }
  for (int l = 0; l < L; l++) {
    n->woff.push_back(n->nw);
    n->nw += (size_t)n->nout[l] * n->kin[l];
  }
  n->nparams = n->nw;
  for (int l = 0; l < L; l++) {
    n->boff.push_back(n->nparams);
    n->nparams += n->nout[l];
  }
  MK(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
  // He-style init of the real entries, zeros in the padding; biases zero.
  std::vector<float> hw(n->nparams, 0.0f);
  std::vector<uint8_t> hm(n->nparams, 0);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < L; l++) {
    const int kr = l == 0 ? in_dim : hidden, nr = l == layers ? out_dim : hidden;
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (float)kr) * (l == layers ? 0.5f : 1.0f));
    for (int r = 0; r < nr; r++)
      for (int c = 0; c < kr; c++) {
        const size_t i = n->woff[l] + (size_t)r * n->kin[l] + c;
        hw[i] = nd(rng);
        hm[i] = 1;
      }
    for (int r = 0; r < nr; r++) hm[n->boff[l] + r] = 1;
  }
  const int Mp = pad128(max_batch);
  MK(cudaMalloc(&n->w, n->nparams * 4));
  MK(cudaMalloc(&n->g, n->nparams * 4));
  MK(cudaMalloc(&n->m, n->nparams * 4));
  MK(cudaMalloc(&n->v, n->nparams * 4));
  MK(cudaMalloc(&n->pmask, n->nparams));
  MK(cudaMemcpy(n->w, hw.data(), n->nparams * 4, cudaMemcpyHostToDevice));
  MK(cudaMemcpy(n->pmask, hm.data(), n->nparams, cudaMemcpyHostToDevice));
  MK(cudaMemset(n->m, 0, n->nparams * 4));
  MK(cudaMemset(n->v, 0, n->nparams * 4));
  size_t tmax = 0;
  for (int l = 0; l < L; l++) {
    bf16 *a = nullptr, *b = nullptr;
    MK(cudaMalloc(&a, (size_t)n->nout[l] * n->kin[l] * 2));
    MK(cudaMalloc(&b, (size_t)n->nout[l] * n->kin[l] * 2));
    n->wt_bf.push_back(a);
    n->w_bf.push_back(b);
    tmax = std::max(tmax, (size_t)std::max(n->kin[l], n->nout[l]));
  }
  for (int l = 0; l < L; l++) {
    bf16* x = nullptr;
    MK(cudaMalloc(&x, (size_t)Mp * n->kin[l] * 2));
    MK(cudaMemset(x, 0, (size_t)Mp * n->kin[l] * 2));
    n->X.push_back(x);
  }
  for (int l = 0; l < L; l++) {
    bf16 *z = nullptr, *d = nullptr;
    MK(cudaMalloc(&z, (size_t)Mp * n->nout[l] * 2));
    MK(cudaMalloc(&d, (size_t)Mp * n->nout[l] * 2));
    n->Z.push_back(z);
    n->dY.push_back(d);
  }
  MK(cudaMalloc(&n->tA, (size_t)Mp * tmax * 2));
  MK(cudaMalloc(&n->tB, (size_t)Mp * tmax * 2));
  MK(cudaMalloc(&n->Y, (size_t)Mp * n->nout[layers] * 4));
  MK(cudaMalloc(&n->loss, 8));
  MK(cudaMalloc(&n->err, 4));
  MK(cudaMemset(n->err, 0, 4));
  int rc = refresh_bf16(n.get());
  if (rc) return rc;
  MK(cudaStreamSynchronize(n->stream));
  *out = n.release();
  set_last_error("");
  return DCFR_OK;
}

void dcfr_mlp_destroy(dcfr_mlp* n) { delete n; }

int dcfr_mlp_num_params(const dcfr_mlp* n, uint64_t* out) {
  if (!n || !out) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *out = n->nparams;
  return DCFR_OK;
}

// Parameters in the padded flat layout (all W_t[l][out][in], then all b[l]).
int dcfr_mlp_get_params(const dcfr_mlp* n, float* host) {
  if (!n || !host) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  MK(cudaMemcpy(host, n->w, n->nparams * 4, cudaMemcpyDeviceToHost));
  return DCFR_OK;
}

int dcfr_mlp_set_params(dcfr_mlp* n, const float* host) {
  if (!n || !host) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  MK(cudaMemcpy(n->w, host, n->nparams * 4, cudaMemcpyHostToDevice));
  int rc = refresh_bf16(n);
  if (rc) return rc;
  MK(cudaStreamSynchronize(n->stream));
  return DCFR_OK;
}

int dcfr_mlp_forward(dcfr_mlp* n, const float* x, int32_t M, float* y) {
  if (!n || !x || !y) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  int rc = batch_ok(n, M);
  if (rc) return rc;
  const int Mp = pad128(M);
  if ((rc = forward(n, x, M, Mp))) return rc;
  const int L = n->layers;
  copy_rows_f32<<<blocks_for((size_t)M * n->out_dim, 256), 256, 0, n->stream>>>(n->Y, n->nout[L], M, n->out_dim, y);
  MK(cudaGetLastError());
  return check_err(n);
}

// Loss and gradients (flat padded layout, host) without updating.
int dcfr_mlp_gradients(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t M, float* loss,
                       float* grads_host) {
  if (!n || !x || !target) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  int rc = batch_ok(n, M);
  if (rc) return rc;
  const int Mp = pad128(M);
  if ((rc = forward(n, x, M, Mp))) return rc;
  if ((rc = backward(n, target, mask, M, Mp))) return rc;
  if ((rc = check_err(n))) return rc;
  if (loss) MK(cudaMemcpy(loss, n->loss, 4, cudaMemcpyDeviceToHost));
  if (grads_host) MK(cudaMemcpy(grads_host, n->g, n->nparams * 4, cudaMemcpyDeviceToHost));
  return DCFR_OK;
}

// One Adam step (beta1 0.9, beta2 0.999, eps 1e-8, bias-corrected) on the
// device gradients times gscale, then the bf16 weight copies.
static int adam_step(dcfr_mlp* n, float lr, float gscale) {
  n->step += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)n->step), c2 = 1.0f - std::pow(b2, (float)n->step);
  adam<<<blocks_for(n->nparams, 256), 256, 0, n->stream>>>(n->w, n->g, n->m, n->v, n->pmask, n->nparams, lr, b1, b2,
                                                           1e-8f, c1, c2, gscale);
  return refresh_bf16(n);
}

int dcfr_mlp_train_step(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t M, float lr,
                        float* loss) {
  if (!n || !x || !target) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  int rc = batch_ok(n, M);
  if (rc) return rc;
  const int Mp = pad128(M);
  if ((rc = forward(n, x, M, Mp))) return rc;
  if ((rc = backward(n, target, mask, M, Mp))) return rc;
  if ((rc = adam_step(n, lr, 1.0f))) return rc;
  if ((rc = check_err(n))) return rc;
  if (loss) MK(cudaMemcpy(loss, n->loss, 4, cudaMemcpyDeviceToHost));
  return DCFR_OK;
}

// Data-parallel training: the loss and gradients of this rank's batch stay
// on the device (the stream is synchronised on return), the caller sums them
// across ranks in place (an all-reduce on dcfr_mlp_gradients_device's
// buffer), then dcfr_mlp_adam_step applies Adam to the sum times gscale.
int dcfr_mlp_backward(dcfr_mlp* n, const float* x, const float* target, const float* mask, int32_t M, float* loss) {
  if (!n || !x || !target) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  int rc = batch_ok(n, M);
  if (rc) return rc;
  const int Mp = pad128(M);
  if ((rc = forward(n, x, M, Mp))) return rc;
  if ((rc = backward(n, target, mask, M, Mp))) return rc;
  if ((rc = check_err(n))) return rc;
  if (loss) MK(cudaMemcpy(loss, n->loss, 4, cudaMemcpyDeviceToHost));
  MK(cudaStreamSynchronize(n->stream));
  return DCFR_OK;
}

int dcfr_mlp_gradients_device(dcfr_mlp* n, float** grads, uint64_t* count) {
  if (!n || !grads || !count) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  *grads = n->g;
  *count = n->nparams;
  return DCFR_OK;
}

int dcfr_mlp_adam_step(dcfr_mlp* n, float lr, float gscale) {
  if (!n) return fail(DCFR_ERR_INVALID_ARG, "NULL argument");
  int rc = adam_step(n, lr, gscale);
  if (rc) return rc;
  if ((rc = check_err(n))) return rc;
  MK(cudaStreamSynchronize(n->stream));
  return DCFR_OK;
}

}  // extern "C"
