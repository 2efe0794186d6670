// CLOUDSC kernels for B200 (sm_100a): FP64 (the reference's double build) and
// FP32-mixed.  One thread walks one column through all levels; all NPROMA
// blocks are processed by one persistent launch (a grid-stride loop over
// column tiles).  See cloudsc_column.cuh for the numerical contract.
//
// Compiled with --fmad=false: no multiply-add contraction, so the FP64 kernel
// performs the reference's operations with one rounding each.
#include <cuda_runtime.h>
#include <cstdint>

#define CSC_DEV __device__ __forceinline__
// Every column of a CTA meets the others at the end of each level, so all
// warps of the CTA run the same stretch of the (very long) level code at the
// same time and share the instruction cache.
#define CSC_LEVEL_SYNC() __syncthreads()
#include "cloudsc_column.cuh"

#include "cloudsc_kparams.h"

namespace cloudsc {

__constant__ KParams<double> c_kpd;
__constant__ KParams<float> c_kpf;
__constant__ KParamsD c_kd;

template <typename Real>
__device__ __forceinline__ const KParams<Real> &KP();
template <>
__device__ __forceinline__ const KParams<double> &KP<double>() { return c_kpd; }
template <>
__device__ __forceinline__ const KParams<float> &KP<float>() { return c_kpf; }

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }
__device__ __forceinline__ void atomic_add(uint32_t *p, uint32_t v) { atomicAdd(p, v); }
__device__ __forceinline__ double xabs(double x) { return fabs(x); }
__device__ __forceinline__ float xabs(float x) { return fabsf(x); }
__device__ __forceinline__ double xsign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float xsign(float a, float b) { return copysignf(a, b); }

}  // namespace cloudsc

#include "cloudsc_body.cuh"

namespace cloudsc {

// Columns are numbered g = ib * NPROMA + jl over all blocks and dealt to CTAs
// in tiles of blockDim.x consecutive columns (a warp reads 32 neighbouring
// columns: coalesced).  The tile loop is uniform over the CTA and every thread
// runs the level loop, so the per-level barrier is reached by all; a thread
// whose column is outside KIDIA..ICEND computes a valid stand-in column and
// stores nothing.
template <bool F32M, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) cloudsc_kernel(Fields F, Shape sh) {
  const long long ncols = (long long)sh.ngpblks * sh.nproma;
  const long long ntiles = (ncols + blockDim.x - 1) / blockDim.x;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long g = tile * blockDim.x + threadIdx.x;
    int ib = (int)(g / sh.nproma);
    int jl = (int)(g - (long long)ib * sh.nproma);
    bool active = ib < sh.ngpblks;
    if (active) active = jl >= sh.kidia0 && jl < min(sh.nproma, sh.ngptot - ib * sh.nproma);
    if (!active) {
      ib = 0;
      jl = sh.kidia0;
    }
    // FP32-mixed: FP32 transcendentals, everything else in double.  (Process
    // rates in float as well were measured at 2.06x the FP64 kernel but with
    // 0.3-4 % tendency errors: float rounding of the rates leaves residues
    // above CLOUDSC's 1e-14 kg/kg thresholds, which switch precipitation
    // processes on and off down the column.)
    cloudsc_column<double, F32M>(F, sh, ib, jl, active);
  }
}

}  // namespace cloudsc

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace cloudsc {

// Upload the parameters to this device's constant memory (all three blocks).
cudaError_t upload_params(const cloudsc_params &p, const Derived &d) {
  KParams<double> kd;
  KParams<float> kf;
  fill_kparams(p, d, kd);
  fill_kparams(p, d, kf);
  KParamsD dd;
  fill_kparams_d(p, dd);
  cudaError_t e = cudaMemcpyToSymbol(c_kpd, &kd, sizeof(kd));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_kpf, &kf, sizeof(kf));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_kd, &dd, sizeof(dd));
  return e;
}

// Register budget and CTA size: __launch_bounds__(MAXT, MINB).  One CTA of
// 448 threads per SM: 14 warps in per-level lock-step at 128 registers (some
// hundred bytes of spills), and 262,144 columns are 586 tiles = 3.96 waves
// over 148 SMs.  Measured at 262,144 columns, FP64: 15.98 ms; 384 threads
// (168 registers) 17.77 ms; 480 threads 16.17 ms; three 128-thread CTAs per
// SM with the same barrier 21.7 ms; no barrier 23.9 ms.
#ifndef CLOUDSC_MAXT
#define CLOUDSC_MAXT 448
#endif
#ifndef CLOUDSC_MINB
#define CLOUDSC_MINB 1
#endif
#ifndef CLOUDSC_MIX_MAXT
#define CLOUDSC_MIX_MAXT 448
#endif
#ifndef CLOUDSC_MIX_MINB
#define CLOUDSC_MIX_MINB 1
#endif

// Largest CTA the kernel of `precision` was compiled for.
int max_threads(int precision) { return precision == 0 ? CLOUDSC_MAXT : CLOUDSC_MIX_MAXT; }

// Launch the kernel: precision 0 = FP64, 1 = FP32-mixed.
cudaError_t launch(int precision, const Fields &f, const Shape &sh, int threads, int grid,
                   cudaStream_t stream) {
  if (precision == 0) {
    if (threads > CLOUDSC_MAXT) return cudaErrorInvalidConfiguration;
    cloudsc_kernel<false, CLOUDSC_MAXT, CLOUDSC_MINB><<<grid, threads, 0, stream>>>(f, sh);
  } else {
    if (threads > CLOUDSC_MIX_MAXT) return cudaErrorInvalidConfiguration;
    cloudsc_kernel<true, CLOUDSC_MIX_MAXT, CLOUDSC_MIX_MINB><<<grid, threads, 0, stream>>>(f, sh);
  }
  return cudaGetLastError();
}

}  // namespace cloudsc

