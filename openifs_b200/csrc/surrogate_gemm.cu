// Column-network GEMMs on the tcgen05 tensor cores (sm_100a).
//
// Activations are row-major [rows][C] bf16 with one row per (column, padded
// level): a column occupies LP consecutive rows, level l at row 2 + l, the
// other rows are zero padding.  A 1-D convolution with 5 taps over levels is
// then five GEMMs whose A operands are the same matrix shifted by -2..+2 rows,
// all accumulated into one TMEM tile:
//
//   D[r][n] = sum_t sum_k A[r + t + tap_origin][k] * W[t][n][k]
//
// TMA fetches each (tap, 64-wide K block) of A (128 rows) and of W (N rows)
// into a 4-stage shared-memory ring; rows outside [0, rows) read as zero.
// Thread 0 issues TMA and tcgen05.mma; the four warps then drain TMEM through
// a fused epilogue (bias, SiLU, residual, padding rows forced to zero, bf16 or
// f32 store; or, for the backward pass, residual gradient and SiLU').
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>
#include <mutex>
#include "tc_gemm.cuh"
#include "cloudsc_surrogate.h"

namespace sg {

constexpr int BM = 128;
constexpr int BK = 64;
constexpr int STAGES = 4;
constexpr int A_BYTES = BM * BK * 2;  // 16 KB

struct Args {
  int rows;        // rows of A and D (tiles past it are masked)
  int kb_per_tap;  // K / 64
  int taps;        // 1 or 5
  int tap_origin;  // row offset of tap 0
  int lp, klev;    // column layout: LP rows per column, levels at rows 2..klev+1
  int epi;
  const float *bias;          // [N] or null
  __nv_bfloat16 *out;         // [rows][N]
  __nv_bfloat16 *out_pre;     // [rows][N] pre-activation (forward) or null
  const __nv_bfloat16 *resid; // [rows][N] residual input (forward) / gradient (backward) or null
  const __nv_bfloat16 *zprev; // [rows][N] pre-activation whose SiLU' scales the gradient (backward)
  __nv_bfloat16 *gout;        // [rows][N] gradient before SiLU' (backward) or null
  float *outf;                // [rows][N] f32 output (linear epilogue)
  unsigned *err;              // or null
};

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + __expf(-z));
  return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ void flag(unsigned *err, unsigned bit) {
  if (err) atomicOr(err, bit);
}

template <int BN, int EPI>
__global__ void __launch_bounds__(128, 1)
    conv_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Args a) {
  constexpr int B_BYTES = BN * BK * 2;
  constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  constexpr uint32_t IDESC = tcg::idesc_bf16_f32(BM, BN);
  constexpr int TMEM_COLS = BN < 32 ? 32 : BN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint64_t *full = (uint64_t *)(smem + STAGES * STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *done = empty + STAGES;
  uint32_t *tmem_slot = (uint32_t *)(done + 1);
  volatile int *abort_flag = (volatile int *)(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tcg::mbar_init(&full[s], 1);
      tcg::mbar_init(&empty[s], 1);
    }
    tcg::mbar_init(done, 1);
    *abort_flag = 0;
    tcg::mbar_fence_init();
    tcg::tma_prefetch_desc(&tmA);
    tcg::tma_prefetch_desc(&tmB);
  }
  if (warp == 0) {
    tcg::tmem_alloc(tmem_slot, TMEM_COLS);
    tcg::tmem_relinquish();
  }
  tcg::tc_fence_before();
  __syncthreads();
  tcg::tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int ntiles = (a.rows + BM - 1) / BM;
  const int nk = a.taps * a.kb_per_tap;
  uint32_t pc = 0, cc = 0;  // produced / consumed stage counters (thread 0)
  uint32_t tile_iter = 0;

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++tile_iter) {
    const int row0 = tile * BM;
    if (tid == 0) {
      bool ok = true;
      auto produce = [&](int k) {
        const int s = pc % STAGES;
        if (pc >= STAGES) ok = ok && tcg::mbar_wait(&empty[s], ((pc / STAGES) - 1) & 1);
        if (!ok) return;
        const int tap = k / a.kb_per_tap, kb = k - tap * a.kb_per_tap;
        uint8_t *sa = smem + s * STAGE_BYTES;
        tcg::mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
        tcg::tma_load_2d(sa, &tmA, &full[s], kb * BK, row0 + a.tap_origin + tap);
        tcg::tma_load_2d(sa + A_BYTES, &tmB, &full[s], kb * BK, tap * BN);
        ++pc;
      };
      const int pre = nk < STAGES - 1 ? nk : STAGES - 1;
      for (int k = 0; k < pre && ok; ++k) produce(k);
      for (int k = 0; k < nk && ok; ++k) {
        const int s = cc % STAGES;
        ok = tcg::mbar_wait(&full[s], (cc / STAGES) & 1);
        if (!ok) break;
        tcg::tc_fence_after();
        const uint32_t sa = tcg::smem_u32(smem + s * STAGE_BYTES);
        const uint64_t da = tcg::sdesc_k_sw128(sa), db = tcg::sdesc_k_sw128(sa + A_BYTES);
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)  // 16 bf16 = 32 bytes per MMA step
          tcg::mma_bf16(tmem, da + 2 * kk, db + 2 * kk, IDESC, (k > 0 || kk > 0) ? 1u : 0u);
        tcg::mma_commit(&empty[s]);
        ++cc;
        if (k + STAGES - 1 < nk) produce(k + STAGES - 1);
      }
      if (ok) {
        tcg::mma_commit(done);
      } else {
        flag(a.err, 1u);
        *abort_flag = 1;
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    if (!tcg::mbar_wait(done, tile_iter & 1)) {
      flag(a.err, 2u);
      *abort_flag = 1;
    }
    tcg::tc_fence_after();

    // ---------------- epilogue: this thread owns output row `row`
    const int row = row0 + warp * 32 + lane;
    const int pos = a.lp > 0 ? row % a.lp : 2;
    const bool in_range = row < a.rows;
    const bool valid = in_range && (a.lp <= 0 || (pos >= 2 && pos < 2 + a.klev));
    if (!*abort_flag) {
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 32) {
        float v[32];
        tcg::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
        if (!in_range) continue;
        const size_t o = (size_t)row * BN + c0;
        if (EPI == CS_EPI_SILU) {
          __align__(16) __nv_bfloat16 h[32], z[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            float zz = v[i] + (a.bias ? a.bias[c0 + i] : 0.0f);
            float hh = silu(zz);
            if (a.resid) hh += __bfloat162float(a.resid[o + i]);
            if (!valid) {
              zz = 0.0f;
              hh = 0.0f;
            }
            z[i] = __float2bfloat16(zz);
            h[i] = __float2bfloat16(hh);
          }
          uint4 *dh = (uint4 *)(a.out + o);
#pragma unroll
          for (int i = 0; i < 4; ++i) dh[i] = ((uint4 *)h)[i];
          if (a.out_pre) {
            uint4 *dz = (uint4 *)(a.out_pre + o);
#pragma unroll
            for (int i = 0; i < 4; ++i) dz[i] = ((uint4 *)z)[i];
          }
        } else if (EPI == CS_EPI_LINEAR_F32) {
          float4 *d = (float4 *)(a.outf + o);
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            float4 w;
            w.x = valid ? v[4 * i + 0] + (a.bias ? a.bias[c0 + 4 * i + 0] : 0.0f) : 0.0f;
            w.y = valid ? v[4 * i + 1] + (a.bias ? a.bias[c0 + 4 * i + 1] : 0.0f) : 0.0f;
            w.z = valid ? v[4 * i + 2] + (a.bias ? a.bias[c0 + 4 * i + 2] : 0.0f) : 0.0f;
            w.w = valid ? v[4 * i + 3] + (a.bias ? a.bias[c0 + 4 * i + 3] : 0.0f) : 0.0f;
            d[i] = w;
          }
        } else {  // CS_EPI_BWD: g = acc (+ residual gradient); dz = g * SiLU'(zprev)
          __align__(16) __nv_bfloat16 g[32], dz[32];
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            float gg = v[i];
            if (a.resid) gg += __bfloat162float(a.resid[o + i]);
            float d = gg * dsilu(__bfloat162float(a.zprev[o + i]));
            if (!valid) {
              gg = 0.0f;
              d = 0.0f;
            }
            g[i] = __float2bfloat16(gg);
            dz[i] = __float2bfloat16(d);
          }
          uint4 *dd = (uint4 *)(a.out + o);
#pragma unroll
          for (int i = 0; i < 4; ++i) dd[i] = ((uint4 *)dz)[i];
          if (a.gout) {
            uint4 *dg = (uint4 *)(a.gout + o);
#pragma unroll
            for (int i = 0; i < 4; ++i) dg[i] = ((uint4 *)g)[i];
          }
        }
      }
    }
    tcg::tc_fence_before();
    __syncthreads();
    if (*abort_flag) break;
  }

  // On an abort, let every copy and MMA this CTA issued land before the
  // shared memory and TMEM are released (bounded waits).
  if (tid == 0 && *abort_flag) {
    for (uint32_t q = cc; q < pc; ++q) (void)tcg::mbar_wait(&full[q % STAGES], (q / STAGES) & 1);
    tcg::mma_commit(done);
    (void)tcg::mbar_wait(done, tile_iter & 1);
  }
  __syncthreads();
  if (warp == 0) tcg::tmem_dealloc(tmem, TMEM_COLS);
}

// ------------------------------------------------------------------ host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  });
  return fn;
}

// Row-major [rows][cols] bf16 matrix, boxes of 64 columns x box_rows rows,
// 128-byte swizzle; out-of-range rows read as zero.
bool make_map(CUtensorMap *m, const void *base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {64, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int BN, int EPI>
cudaError_t launch_t(const CUtensorMap &ma, const CUtensorMap &mb, const Args &a, int grid, cudaStream_t st) {
  const int smem = STAGES * (A_BYTES + BN * BK * 2) + 1024 + 256;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e =
        cudaFuncSetAttribute(conv_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  conv_gemm_kernel<BN, EPI><<<grid, 128, smem, st>>>(ma, mb, a);
  return cudaGetLastError();
}

}  // namespace sg

extern "C" int cs_conv_gemm(const cs_gemm_desc *g, void *stream) {
  using namespace sg;
  if (!g || !g->a || !g->w) return CS_E_ARG;
  if (g->k % 64 || g->k <= 0 || (g->n != 64 && g->n != 128) || (g->taps != 1 && g->taps != 5) ||
      g->rows <= 0)
    return CS_E_ARG;
  if (g->epi < CS_EPI_SILU || g->epi > CS_EPI_BWD) return CS_E_ARG;
  if (g->epi == CS_EPI_LINEAR_F32 ? !g->outf : !g->out) return CS_E_ARG;
  if (g->epi == CS_EPI_BWD && !g->zprev) return CS_E_ARG;
  if (((uintptr_t)g->a | (uintptr_t)g->w | (uintptr_t)g->out | (uintptr_t)g->out_pre | (uintptr_t)g->gout |
       (uintptr_t)g->outf) &
      15)
    return CS_E_ARG;
  CUtensorMap ma, mb;
  if (!make_map(&ma, g->a, (uint64_t)g->rows, (uint64_t)g->k, BM)) return CS_E_CUDA;
  if (!make_map(&mb, g->w, (uint64_t)g->taps * g->n, (uint64_t)g->k, (uint32_t)g->n)) return CS_E_CUDA;
  Args a;
  memset(&a, 0, sizeof(a));
  a.rows = g->rows;
  a.kb_per_tap = g->k / 64;
  a.taps = g->taps;
  a.tap_origin = g->taps == 5 ? -2 : 0;
  a.lp = g->lp;
  a.klev = g->klev;
  a.epi = g->epi;
  a.bias = g->bias;
  a.out = (__nv_bfloat16 *)g->out;
  a.out_pre = (__nv_bfloat16 *)g->out_pre;
  a.resid = (const __nv_bfloat16 *)g->resid;
  a.zprev = (const __nv_bfloat16 *)g->zprev;
  a.gout = (__nv_bfloat16 *)g->gout;
  a.outf = g->outf;
  a.err = g->err;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int ntiles = (g->rows + BM - 1) / BM;
  const int grid = ntiles < sms ? ntiles : sms;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (g->n == 128) {
    if (g->epi == CS_EPI_SILU) e = launch_t<128, CS_EPI_SILU>(ma, mb, a, grid, st);
    else if (g->epi == CS_EPI_BWD) e = launch_t<128, CS_EPI_BWD>(ma, mb, a, grid, st);
    else e = launch_t<128, CS_EPI_LINEAR_F32>(ma, mb, a, grid, st);
  } else {
    if (g->epi == CS_EPI_SILU) e = launch_t<64, CS_EPI_SILU>(ma, mb, a, grid, st);
    else if (g->epi == CS_EPI_BWD) e = launch_t<64, CS_EPI_BWD>(ma, mb, a, grid, st);
    else e = launch_t<64, CS_EPI_LINEAR_F32>(ma, mb, a, grid, st);
  }
  return e == cudaSuccess ? CS_OK : CS_E_CUDA;
}
