// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05) for
// the leaf-value network (mlp.cu):
//
//   C[M][N] = epilogue( sum_k A[M][K] * B[N][K] )
//
// A and B are row-major with K contiguous (both operands "K-major"). One CTA
// computes a 128 x 128 tile of C:
//   * warp 0, one thread: TMA loads of 128 x 64 tiles of A and B into a
//     GEMM_STAGES-deep shared-memory ring (128-byte swizzle, the canonical
//     K-major layout the tensor core reads);
//   * warp 1, one thread: tcgen05.mma (M=128, N=128, K=16 per instruction,
//     FP32 accumulator in tensor memory), a tcgen05.commit per stage frees
//     the stage, a last commit marks the accumulator complete;
//   * all four warps: the epilogue reads the accumulator with tcgen05.ld
//     (warp w owns rows 32w..32w+31) and writes C through the epilogue.
// Every wait on an mbarrier is bounded; a wait that gives up records an error
// code and the CTA skips the rest of its work, frees its tensor memory and
// returns.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace dcfr {

// Two CTAs per SM (a 3-stage ring each, 97 KB of shared memory and 128
// tensor-memory columns): one CTA's epilogue runs under the other's MMAs,
// and a 4096 x 1024 output (256 tiles) fits the 148 SMs in one wave.
#ifndef GEMM_STAGES_CFG
#define GEMM_STAGES_CFG 3
#endif
#ifndef GEMM_CTAS_PER_SM
#define GEMM_CTAS_PER_SM 2
#endif
constexpr int GEMM_BM = 128, GEMM_BN = 128, GEMM_BK = 64, GEMM_STAGES = GEMM_STAGES_CFG, GEMM_THREADS = 128;
constexpr uint32_t GEMM_TILE_BYTES = GEMM_BM * GEMM_BK * 2;  // one 128 x 64 bf16 tile
constexpr size_t GEMM_SMEM = 1024 + 2 * GEMM_STAGES * (size_t)GEMM_TILE_BYTES + 256;
constexpr long long GEMM_WAIT_LIMIT = 1ll << 22;  // polls before a wait gives up (well over a second)

// Epilogues.
enum GemmEpi : int {
  EPI_F32 = 0,            // C (f32) = acc
  EPI_BIAS_F32 = 1,       // C (f32) = acc + bias[n]
  EPI_BIAS_GELU = 2,      // Z (bf16) = acc + bias[n]; C (bf16) = gelu(acc + bias[n])
  EPI_GELU_GRAD = 3,      // C (bf16) = acc * gelu'(Z[m][n])
};

struct GemmArgs {
  void* c;               // f32 or bf16 output [M][ldc]
  __nv_bfloat16* z;      // EPI_BIAS_GELU: pre-activation out; EPI_GELU_GRAD: pre-activation in
  const float* bias;     // [N]
  int ldc;
  int epi;
  int M, N, K;
  int* error;            // set to a nonzero code when a bounded wait gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false if the barrier did not complete the phase in time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (long long i = 0; i < GEMM_WAIT_LIMIT; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor (tcgen05): K-major, 128-byte swizzle,
// 8-row groups 1024 bytes apart.
__device__ __forceinline__ uint64_t sw128_desc(const void* p) {
  const uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr & 0x3FFFF) >> 4;       // start address [0,14)
  d |= (uint64_t)1 << 16;           // leading byte offset (unused for swizzled K-major), [16,30)
  d |= (uint64_t)(1024 >> 4) << 32; // stride byte offset [32,46)
  d |= (uint64_t)1 << 46;           // descriptor version [46,48)
  d |= (uint64_t)2 << 61;           // layout: 128-byte swizzle [61,64)
  return d;
}

// Instruction descriptor: kind::f16, BF16 A and B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int m, int n) {
  return (1u << 4)                     // D format F32
         | (1u << 7)                   // A format BF16
         | (1u << 10)                  // B format BF16
         | ((uint32_t)(n >> 3) << 17)  // N >> 3
         | ((uint32_t)(m >> 4) << 24); // M >> 4
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.3989422804014327f * expf(-0.5f * x * x);
}

__global__ void __launch_bounds__(GEMM_THREADS, GEMM_CTAS_PER_SM)
    gemm_bf16_tc_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                        GemmArgs G) {
  extern __shared__ __align__(1024) unsigned char gemm_smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(((uintptr_t)gemm_smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sa = smem;
  unsigned char* sb = smem + GEMM_STAGES * GEMM_TILE_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + 2 * GEMM_STAGES * GEMM_TILE_BYTES);
  uint64_t* empty = full + GEMM_STAGES;
  uint64_t* accf = empty + GEMM_STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accf + 1);
  __shared__ int failed;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * GEMM_BM, n0 = blockIdx.x * GEMM_BN;
  const int nk = G.K / GEMM_BK;

  if (tid == 0) {
    failed = 0;
    for (int s = 0; s < GEMM_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(GEMM_BN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // Producer.
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % GEMM_STAGES;
      if (kb >= GEMM_STAGES && !mbar_wait(&empty[s], ((kb / GEMM_STAGES) - 1) & 1)) {
        failed = 1;
        break;
      }
      mbar_expect_tx(&full[s], 2 * GEMM_TILE_BYTES);
      tma_load_2d(sa + s * GEMM_TILE_BYTES, &map_a, &full[s], kb * GEMM_BK, m0);
      tma_load_2d(sb + s * GEMM_TILE_BYTES, &map_b, &full[s], kb * GEMM_BK, n0);
    }
  } else if (warp == 1 && lane == 0) {
    // Tensor-core issue.
    const uint32_t idesc = idesc_bf16_f32(GEMM_BM, GEMM_BN);
    for (int kb = 0; kb < nk; kb++) {
      const int s = kb % GEMM_STAGES;
      if (!mbar_wait(&full[s], (kb / GEMM_STAGES) & 1)) {
        failed = 2;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint64_t da = sw128_desc(sa + s * GEMM_TILE_BYTES), db = sw128_desc(sb + s * GEMM_TILE_BYTES);
#pragma unroll
      for (int k = 0; k < GEMM_BK / 16; k++)  // K = 16 per instruction: 32 bytes along the swizzled row
        umma_bf16(tmem, da + (uint64_t)(2 * k), db + (uint64_t)(2 * k), idesc, (kb > 0 || k > 0) ? 1u : 0u);
      umma_commit(&empty[s]);
    }
    umma_commit(accf);
  }
  __syncwarp();
  // Epilogue: every thread owns one row of the tile.
  const bool ok = mbar_wait(accf, 0);
  if (!ok && lane == 0) atomicExch(&failed, 3);
  __syncwarp();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // tcgen05.ld is warp-collective: decide once per warp.
  const bool go = __all_sync(0xffffffffu, ok && *(volatile int*)&failed == 0);
  if (go) {
    const int m = m0 + warp * 32 + lane;
    const uint32_t row_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < GEMM_BN; c0 += 32) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
          "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
            "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
          : "r"(row_addr + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < G.M) {
        const int nb = n0 + c0;
        if (G.epi == EPI_F32 || G.epi == EPI_BIAS_F32) {
          float* out = reinterpret_cast<float*>(G.c) + (size_t)m * G.ldc + nb;
#pragma unroll
          for (int j = 0; j < 32; j += 4) {
            float4 o;
            o.x = __uint_as_float(v[j]) + (G.epi == EPI_BIAS_F32 ? G.bias[nb + j] : 0.0f);
            o.y = __uint_as_float(v[j + 1]) + (G.epi == EPI_BIAS_F32 ? G.bias[nb + j + 1] : 0.0f);
            o.z = __uint_as_float(v[j + 2]) + (G.epi == EPI_BIAS_F32 ? G.bias[nb + j + 2] : 0.0f);
            o.w = __uint_as_float(v[j + 3]) + (G.epi == EPI_BIAS_F32 ? G.bias[nb + j + 3] : 0.0f);
            *reinterpret_cast<float4*>(out + j) = o;
          }
        } else {
          __nv_bfloat16* out = reinterpret_cast<__nv_bfloat16*>(G.c) + (size_t)m * G.ldc + nb;
          __nv_bfloat16* zz = G.z + (size_t)m * G.ldc + nb;
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            float a = __uint_as_float(v[j]), b = __uint_as_float(v[j + 1]);
            __nv_bfloat162 r;
            if (G.epi == EPI_BIAS_GELU) {
              a += G.bias[nb + j];
              b += G.bias[nb + j + 1];
              *reinterpret_cast<__nv_bfloat162*>(zz + j) = __floats2bfloat162_rn(a, b);
              r = __floats2bfloat162_rn(gelu(a), gelu(b));
            } else {
              const __nv_bfloat162 zv = *reinterpret_cast<const __nv_bfloat162*>(zz + j);
              r = __floats2bfloat162_rn(a * gelu_grad(__bfloat162float(zv.x)), b * gelu_grad(__bfloat162float(zv.y)));
            }
            *reinterpret_cast<__nv_bfloat162*>(out + j) = r;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (failed && tid == 0 && G.error) atomicExch(G.error, failed);
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(GEMM_BN) : "memory");
  }
}

}  // namespace dcfr
