// Shared helpers for the holotomo B200 kernels: complex arithmetic, error
// reporting, and the per-size twiddle tables.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>

namespace ht {

// ----------------------------------------------------------------- errors
// Thread-local last-error message (read through ht_last_error()).
void set_error(const std::string& msg);
const char* last_error();

#define HT_CHECK_CUDA(expr)                                                     \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess) {                                                    \
      ::ht::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));      \
      return 2;                                                                 \
    }                                                                           \
  } while (0)

#define HT_REQUIRE(cond, msg)                                                   \
  do {                                                                          \
    if (!(cond)) {                                                              \
      ::ht::set_error(msg);                                                     \
      return 1;                                                                 \
    }                                                                           \
  } while (0)

// Status codes returned by every entry point.
enum Status : int { kOk = 0, kBadArgument = 1, kCudaError = 2, kUnsupported = 3 };

// ------------------------------------------------------------ complex math
// On the device the two parts of a complex value go through one packed
// two-lane FP32 instruction (add/sub/mul/fma .f32x2, sm_100): the same IEEE
// operation on each part as the scalar forms, in half the instructions
// (cmul/cmulc stay scalar: their lane swaps cost more than they save).  A
// translation unit that defines HT_SCALAR_COMPLEX before including this
// keeps scalar adds and scales (the column passes of prop.cu run faster so).
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float2 p2_add(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 pa, pb, pd;\n mov.b64 pa, {%2, %3};\n mov.b64 pb, {%4, %5};\n add.rn.f32x2 pd, pa, pb;\n"
      " mov.b64 {%0, %1}, pd;\n}" : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 p2_sub(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 pa, pb, pd;\n mov.b64 pa, {%2, %3};\n mov.b64 pb, {%4, %5};\n sub.rn.f32x2 pd, pa, pb;\n"
      " mov.b64 {%0, %1}, pd;\n}" : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 p2_mul(float2 a, float2 b) {
  float2 d;
  asm("{\n .reg .b64 pa, pb, pd;\n mov.b64 pa, {%2, %3};\n mov.b64 pb, {%4, %5};\n mul.rn.f32x2 pd, pa, pb;\n"
      " mov.b64 {%0, %1}, pd;\n}" : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
// a * b + c, lane by lane
__device__ __forceinline__ float2 p2_fma(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{\n .reg .b64 pa, pb, pc, pd;\n mov.b64 pa, {%2, %3};\n mov.b64 pb, {%4, %5};\n mov.b64 pc, {%6, %7};\n"
      " fma.rn.f32x2 pd, pa, pb, pc;\n mov.b64 {%0, %1}, pd;\n}"
      : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
#endif

__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && !defined(HT_SCALAR_COMPLEX)
  return p2_add(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__) && !defined(HT_SCALAR_COMPLEX)
  return p2_sub(a, b);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) {
#if defined(__CUDA_ARCH__) && !defined(HT_SCALAR_COMPLEX)
  return p2_mul(a, make_float2(s, s));
#else
  return make_float2(a.x * s, a.y * s);
#endif
}
// multiply by -i (forward sign) or +i (inverse sign)
template <bool INV>
__host__ __device__ __forceinline__ float2 rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
__host__ __device__ __forceinline__ float2 cmul_i(float2 a) { return make_float2(-a.y, a.x); }  // i*a

// Bulk prefetch of [p, p + bytes) into L2 by the TMA unit: one instruction, no
// registers, no shared memory and nothing to wait for; a kernel issues it for
// rows it reads only later, so that those loads hit L2.  Skipped unless p is
// 16-byte aligned and bytes a multiple of 16 (the instruction's rules); the
// whole range must lie inside one allocation.
__device__ __forceinline__ void l2_prefetch(const void* p, unsigned bytes) {
#if defined(__CUDA_ARCH__)
  if ((reinterpret_cast<unsigned long long>(p) & 15ull) == 0ull && (bytes & 15u) == 0u)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
#endif
}

// --------------------------------------------------------- twiddle tables
// For every supported transform length N the library keeps, per device, a
// table tw4[m] = exp(-2*pi*i*m/(4N)), m in [0, 4N), computed in double and
// rounded once.  FFT twiddles W_N^a are tw4[4a]; the DCT pre/post twiddles
// exp(-i*pi*k/(2N)) are tw4[k].
const float2* twiddle_table(int N, int device);  // nullptr + error on failure

// Number of kernels this library has launched (read through ht_launch_count()).
void count_launch();
long launch_count();

// Per-kernel CUDA-event timers (read through ht_ktimer_*).  A KTimer around a
// launch records an event pair on the launch stream when the kernel's timer
// is armed and the stream is not being captured into a graph; `units` is the
// work of the launch (images, or slices for the Radon kernels).
struct KTimer {
  int slot = -1;
  cudaStream_t st = nullptr;
  KTimer(const char* name, cudaStream_t stream, double units);
  ~KTimer();
};

// Sizes accepted by the line transforms: N = 2^a 3^b from the list below.
bool fft_size_supported(int N);

}  // namespace ht
