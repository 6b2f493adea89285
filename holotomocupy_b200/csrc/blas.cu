// BLAS-1 for the BH updates (reference: Chunking.linear_batch /
// linear_redot_batch / redot_batch, src/holotomocupy/chunking.py:235-290, and
// utils.redot, src/holotomocupy/utils.py:96-104).  Arrays are viewed as
// float32 vectors (complex64 = interleaved pairs); inner products are
// accumulated in double precision (the reference accumulates in float32).
#include "common.cuh"
#include "holotomo_b200_internal.h"

namespace ht {

constexpr int kBlasThreads = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[kBlasThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < kBlasThreads / 32; ++i) s += red[i];
  return s;
}

// x = a x + b y;  if dot: *dot += sum y * x_new
template <bool DOT>
__device__ __forceinline__ void axpby_body(float* __restrict__ x, const float* __restrict__ y, float a, float b, long n,
                                           double* __restrict__ dot) {
  double acc = 0.0;
  const long n4 = n / 4;
  float4* x4 = reinterpret_cast<float4*>(x);
  const float4* y4 = reinterpret_cast<const float4*>(y);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    float4 xv = x4[i];
    const float4 yv = y4[i];
    xv.x = a * xv.x + b * yv.x;
    xv.y = a * xv.y + b * yv.y;
    xv.z = a * xv.z + b * yv.z;
    xv.w = a * xv.w + b * yv.w;
    x4[i] = xv;
    if (DOT) acc += (double)(yv.x * xv.x + yv.y * xv.y) + (double)(yv.z * xv.z + yv.w * xv.w);
  }
  if (blockIdx.x == 0)
    for (long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) {
      x[i] = a * x[i] + b * y[i];
      if (DOT) acc += (double)(y[i] * x[i]);
    }
  if (DOT) {
    const double s = block_sum(acc);
    if (threadIdx.x == 0) atomicAdd(dot, s);
  }
}

template <bool DOT>
__global__ void __launch_bounds__(kBlasThreads) k_axpby(float* __restrict__ x, const float* __restrict__ y, float a,
                                                        float b, long n, double* __restrict__ dot) {
  axpby_body<DOT>(x, y, a, b, n, dot);
}

// The same with a = (float)(*A) * sa, b = (float)(*B) * sb read on the device
// (A or B null: the factor alone), so the step sizes never visit the host.
template <bool DOT>
__global__ void __launch_bounds__(kBlasThreads) k_axpby_dev(float* __restrict__ x, const float* __restrict__ y,
                                                            const double* __restrict__ A, float sa,
                                                            const double* __restrict__ B, float sb, long n,
                                                            double* __restrict__ dot) {
  const float a = A ? (float)(*A) * sa : sa;
  const float b = B ? (float)(*B) * sb : sb;
  axpby_body<DOT>(x, y, a, b, n, dot);
}

// Step sizes of one BH iteration (rec_mpi.py:180-218) from the Hessian forms
// H = {H(g,g), H_ref(g,eta), H(eta,eta), H_sym(g,eta)} and the inner products
// dots = {<eta,g>_obj, <eta,g>_pos, <eta,g>_prb} of the new direction.
// phase 0: scal[0] = beta = first ? 0 : H[1] / H[2].
// phase 1: scal[1] = alpha = top / bottom with
//   top = -(dots[0]/rho_obj + dots[1]/rho_pos + dots[2]/rho_prb),
//   bottom = first ? H[0] : beta^2 H[2] - 2 beta H[3] + H[0];
//   (alpha, beta) is appended to hist[*count] while *count < cap.
__global__ void k_bh_scalars(const double* __restrict__ H, double* __restrict__ dots, int first, int phase,
                             double rho_obj, double rho_pos, double rho_prb, double* __restrict__ scal,
                             double* __restrict__ hist, int cap, int* __restrict__ count) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (phase == 0) {
    scal[0] = first ? 0.0 : H[1] / H[2];
    if (dots)  // the direction updates that follow accumulate into them
      for (int i = 0; i < 3; ++i) dots[i] = 0.0;
    return;
  }
  const double beta = scal[0];
  const double top = -(dots[0] / rho_obj + dots[1] / rho_pos + dots[2] / rho_prb);
  const double bottom = first ? H[0] : beta * beta * H[2] - 2.0 * beta * H[3] + H[0];
  const double alpha = top / bottom;
  scal[1] = alpha;
  if (hist && count) {
    const int i = *count;
    if (i < cap) {
      hist[2 * i + 0] = alpha;
      hist[2 * i + 1] = beta;
    }
    *count = i + 1;
  }
}

__global__ void __launch_bounds__(kBlasThreads) k_dot(const float* __restrict__ x, const float* __restrict__ y, long n,
                                                      double* __restrict__ dot) {
  double acc = 0.0;
  const long n4 = n / 4;
  const float4* x4 = reinterpret_cast<const float4*>(x);
  const float4* y4 = reinterpret_cast<const float4*>(y);
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long)gridDim.x * blockDim.x) {
    const float4 xv = x4[i], yv = y4[i];
    acc += (double)(xv.x * yv.x + xv.y * yv.y) + (double)(xv.z * yv.z + xv.w * yv.w);
  }
  if (blockIdx.x == 0)
    for (long i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) acc += (double)(x[i] * y[i]);
  const double s = block_sum(acc);
  if (threadIdx.x == 0) atomicAdd(dot, s);
}

static unsigned blas_grid(long n) {
  long g = (n / 4 + kBlasThreads - 1) / kBlasThreads;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace ht

extern "C" int ht_axpby(void* x, const void* y, float a, float b, long n, double* dot, void* stream) {
  using namespace ht;
  HT_REQUIRE(x && y, "ht_axpby: null pointer");
  HT_REQUIRE(((uintptr_t)x % 16 == 0) && ((uintptr_t)y % 16 == 0), "ht_axpby: arrays must be 16-byte aligned");
  if (n == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dot) {
    k_axpby<true><<<blas_grid(n), kBlasThreads, 0, st>>>((float*)x, (const float*)y, a, b, n, dot);
    ::ht::count_launch();
  }
  else {
    k_axpby<false><<<blas_grid(n), kBlasThreads, 0, st>>>((float*)x, (const float*)y, a, b, n, nullptr);
    ::ht::count_launch();
  }
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_dot(const void* x, const void* y, long n, double* dot, void* stream) {
  using namespace ht;
  HT_REQUIRE(x && y && dot, "ht_dot: null pointer");
  HT_REQUIRE(((uintptr_t)x % 16 == 0) && ((uintptr_t)y % 16 == 0), "ht_dot: arrays must be 16-byte aligned");
  if (n == 0) return kOk;
  k_dot<<<blas_grid(n), kBlasThreads, 0, static_cast<cudaStream_t>(stream)>>>((const float*)x, (const float*)y, n,
                                                                             dot); ::ht::count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_axpby_dev(void* x, const void* y, const double* A, float sa, const double* B, float sb, long n,
                            double* dot, void* stream) {
  using namespace ht;
  HT_REQUIRE(x && y, "ht_axpby_dev: null pointer");
  HT_REQUIRE(((uintptr_t)x % 16 == 0) && ((uintptr_t)y % 16 == 0), "ht_axpby_dev: arrays must be 16-byte aligned");
  if (n == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dot)
    k_axpby_dev<true><<<blas_grid(n), kBlasThreads, 0, st>>>((float*)x, (const float*)y, A, sa, B, sb, n, dot);
  else
    k_axpby_dev<false><<<blas_grid(n), kBlasThreads, 0, st>>>((float*)x, (const float*)y, A, sa, B, sb, n, nullptr);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_bh_scalars(const double* H, double* dots, int first, int phase, double rho_obj,
                             double rho_pos, double rho_prb, double* scal, double* hist, int cap, int* count,
                             void* stream) {
  using namespace ht;
  HT_REQUIRE(H && scal, "ht_bh_scalars: null pointer");
  HT_REQUIRE(phase == 0 || phase == 1, "ht_bh_scalars: phase must be 0 or 1");
  HT_REQUIRE(phase == 0 || dots, "ht_bh_scalars: phase 1 needs dots");
  HT_REQUIRE(cap >= 0 && (!hist || count), "ht_bh_scalars: hist needs count");
  k_bh_scalars<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(H, dots, first, phase, rho_obj, rho_pos, rho_prb,
                                                                 scal, hist, cap, count);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}
