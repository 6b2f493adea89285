// 3-D Laplacian regulariser of the BH functional (reference:
// src/holotomocupy/rec_mpi.py:402-496).
//
// L is the 7-point Laplacian, periodic in y and x (cp.roll) and applied to the
// object zero-padded by two slices in z.  The reference's gradient and
// Hessian form use B = L o L where the inner L is evaluated on the object
// slices and on the ghost slice next to each end (rec_mpi.py:437-440); its
// energy uses the inner L on the object slices only (rec_mpi.py:486-493).
//   k_lap_ext:   lap[ze] = (L u~)(ze - 1), ze in [0, nz + 2)   (u~: zero outside [0, nz))
//   k_lap_apply: (B u)(z) = lap[z] + lap[z + 2] + in-plane neighbours of lap[z + 1] - 6 lap[z + 1],
//                then g += s * B u, or the per-block double-precision partials of Re<y, B u>,
//                which k_lap_finish adds in block order (the sums repeat bit for bit).
// The sums keep the reference's order a + c + b[y+1] + b[y-1] + b[x+1] + b[x-1] - 6 b.
#include <algorithm>

#include "common.cuh"
#include "holotomo_b200_internal.h"

namespace ht {

template <class T>
struct RE;
template <>
struct RE<float2> {
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
  static __device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
  static __device__ __forceinline__ float2 scale(float2 a, float s) { return make_float2(s * a.x, s * a.y); }
  static __device__ __forceinline__ double redot(float2 a, float2 b) { return (double)(a.x * b.x + a.y * b.y); }
};
template <>
struct RE<float> {
  static __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
  static __device__ __forceinline__ float scale(float a, float s) { return s * a; }
  static __device__ __forceinline__ double redot(float a, float b) { return (double)(a * b); }
};

// a + c + b[y+1] + b[y-1] + b[x+1] + b[x-1] - 6 b  (rec_mpi.py:432-436)
template <class T>
__device__ __forceinline__ T lap7(T a, T c, T byp, T bym, T bxp, T bxm, T b) {
  T v = RE<T>::add(a, c);
  v = RE<T>::add(v, byp);
  v = RE<T>::add(v, bym);
  v = RE<T>::add(v, bxp);
  v = RE<T>::add(v, bxm);
  return RE<T>::sub(v, RE<T>::scale(b, 6.f));
}

// The kernels walk rows (z, y) of the volume, the threads of a CTA across x,
// so a row's indices are formed once per row rather than divided out of a
// flat index per element.
template <class T>
__global__ void __launch_bounds__(256) k_lap_ext(const T* __restrict__ u, T* __restrict__ lap, int nz, int ny, int nx) {
  const int nrows = (nz + 2) * ny;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int ze = r / ny, y = r - ze * ny;
    const int z = ze - 1;
    const int yp = (y + 1 == ny) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
    auto U = [&](int zz, int yy, int xx) -> T {
      return (zz < 0 || zz >= nz) ? RE<T>::zero() : __ldg(&u[((long)zz * ny + yy) * nx + xx]);
    };
    T* out = lap + (long)r * nx;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const int xp = (x + 1 == nx) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
      out[x] = lap7(U(z - 1, y, x), U(z + 1, y, x), U(z, yp, x), U(z, ym, x), U(z, y, xp), U(z, y, xm), U(z, y, x));
    }
  }
}

constexpr int kRegThreads = 256;

template <class T, int MODE>
__global__ void __launch_bounds__(kRegThreads)
k_lap_apply(const T* __restrict__ lap, int nz, int ny, int nx, float s, T* __restrict__ g, const T* __restrict__ yv,
            double* __restrict__ out, const T* __restrict__ yv2) {
  const long plane = (long)ny * nx;
  const int nrows = nz * ny;
  double acc = 0.0, acc2 = 0.0;
  for (int r = blockIdx.x; r < nrows; r += gridDim.x) {
    const int z = r / ny, y = r - z * ny;
    const int yp = (y + 1 == ny) ? 0 : y + 1, ym = (y == 0) ? ny - 1 : y - 1;
    const T* b = lap + (long)(z + 1) * plane;
    const long row = (long)r * nx;
    for (int x = threadIdx.x; x < nx; x += blockDim.x) {
      const int xp = (x + 1 == nx) ? 0 : x + 1, xm = (x == 0) ? nx - 1 : x - 1;
      const long i = row + x;
      const T v = lap7(__ldg(&lap[(long)z * plane + (long)y * nx + x]),
                       __ldg(&lap[(long)(z + 2) * plane + (long)y * nx + x]), __ldg(&b[(long)yp * nx + x]),
                       __ldg(&b[(long)ym * nx + x]), __ldg(&b[(long)y * nx + xp]), __ldg(&b[(long)y * nx + xm]),
                       __ldg(&b[(long)y * nx + x]));
      if (MODE == 0) {
        g[i] = RE<T>::add(g[i], RE<T>::scale(v, s));
      } else {
        acc += RE<T>::redot(__ldg(&yv[i]), v);
        if (yv2) acc2 += RE<T>::redot(__ldg(&yv2[i]), v);
      }
    }
  }
  if (MODE == 1) {
    __shared__ double red[2][kRegThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_down_sync(0xffffffffu, acc, o);
      acc2 += __shfl_down_sync(0xffffffffu, acc2, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red[0][threadIdx.x / 32] = acc;
      red[1][threadIdx.x / 32] = acc2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0, t2 = 0.0;
      for (int w = 0; w < kRegThreads / 32; ++w) {
        t += red[0][w];
        t2 += red[1][w];
      }
      out[2 * blockIdx.x] = t;   // out: the per-block partials (k_lap_finish adds them)
      out[2 * blockIdx.x + 1] = t2;
    }
  }
}

// the per-block partials (out[2 b]) of the sum over the object slices of |lap|^2
template <class T>
__global__ void __launch_bounds__(kRegThreads)
k_lap_energy(const T* __restrict__ lap, long n, double* __restrict__ out) {
  double acc = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const T v = __ldg(&lap[i]);
    acc += RE<T>::redot(v, v);
  }
  __shared__ double red[kRegThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRegThreads / 32; ++w) t += red[w];
    out[2 * blockIdx.x] = t;   // out: the per-block partials (k_lap_finish adds them)
  }
}

// *out += sd * (the partials part[2 b] summed), and the same for out2 with
// part[2 b + 1], by one warp: lane l sums blocks l, l + 32, ... and the lanes
// combine in a fixed shuffle tree, so the sums repeat bit for bit
__global__ void k_lap_finish(const double* __restrict__ part, int nblk, double sd, double* __restrict__ out,
                             double* __restrict__ out2) {
  double t = 0.0, t2 = 0.0;
  for (int b = threadIdx.x; b < nblk; b += 32) {
    t += part[2 * b];
    if (out2) t2 += part[2 * b + 1];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    t += __shfl_down_sync(0xffffffffu, t, o);
    t2 += __shfl_down_sync(0xffffffffu, t2, o);
  }
  if (threadIdx.x == 0) {
    *out += sd * t;
    if (out2) *out2 += sd * t2;
  }
}

// Per-block partial sums of the forms and the energy sit after the extended
// Laplacian in the workspace, at the next 16-byte boundary: at most
// kRegMaxBlocks blocks, two doubles each, within the 64 KiB reserved there.
constexpr long kRegMaxBlocks = 148L * 16;
constexpr long kLapPartBytes = 64 * 1024;
static_assert(kRegMaxBlocks * 2 * (long)sizeof(double) <= kLapPartBytes, "partial sums exceed their area");
static double* lap_partials(void* work, int nz, int ny, int nx, int is_complex) {
  const long off = ((long)(nz + 2) * ny * nx * (is_complex ? 8 : 4) + 15) / 16 * 16;
  return reinterpret_cast<double*>(static_cast<char*>(work) + off);
}

// k_lap_apply's grid: CTAs over the rows (z, y) of the volume
static unsigned reg_grid_rows(int nz, int ny) {
  const long rows = (long)nz * ny;
  return (unsigned)std::max<long>(1, std::min<long>(rows, kRegMaxBlocks));
}

static unsigned reg_grid(long n) {
  long g = (n + kRegThreads - 1) / kRegThreads;
  if (g > kRegMaxBlocks) g = kRegMaxBlocks;
  return (unsigned)(g < 1 ? 1 : g);
}

template <class T>
static cudaError_t lap_ext(const void* u, void* work, int nz, int ny, int nx, cudaStream_t st) {
  const long rows = (long)(nz + 2) * ny;
  k_lap_ext<T><<<(unsigned)std::min<long>(rows, 148L * 32), 256, 0, st>>>(static_cast<const T*>(u),
                                                                          static_cast<T*>(work), nz, ny, nx);
  count_launch();
  return cudaGetLastError();
}

}  // namespace ht

#define HT_REG_CHECK(name)                                                                 \
  HT_REQUIRE(nz > 0 && ny > 0 && nx > 0, name ": sizes must be positive");                 \
  HT_REQUIRE(work != nullptr, name ": null workspace")

extern "C" int ht_laplacian_grad(const void* u, void* g, int nz, int ny, int nx, int is_complex, float scale,
                                 void* work, void* stream) {
  using namespace ht;
  HT_REQUIRE(u && g, "ht_laplacian_grad: null pointer");
  HT_REG_CHECK("ht_laplacian_grad");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned rows = reg_grid_rows(nz, ny);
  if (is_complex) {
    HT_CHECK_CUDA(lap_ext<float2>(u, work, nz, ny, nx, st));
    k_lap_apply<float2, 0><<<rows, kRegThreads, 0, st>>>(static_cast<const float2*>(work), nz, ny, nx, scale,
                                                         static_cast<float2*>(g), nullptr, nullptr, nullptr);
  } else {
    HT_CHECK_CUDA(lap_ext<float>(u, work, nz, ny, nx, st));
    k_lap_apply<float, 0><<<rows, kRegThreads, 0, st>>>(static_cast<const float*>(work), nz, ny, nx, scale,
                                                        static_cast<float*>(g), nullptr, nullptr, nullptr);
  }
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_laplacian_dot(const void* y, const void* z, int nz, int ny, int nx, int is_complex, double scale,
                                void* work, double* out, const void* y2, double* out2, void* stream) {
  using namespace ht;
  HT_REQUIRE(y && z && out, "ht_laplacian_dot: null pointer");
  HT_REQUIRE(!y2 || out2, "ht_laplacian_dot: y2 needs out2");
  HT_REG_CHECK("ht_laplacian_dot");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const unsigned rows = reg_grid_rows(nz, ny);
  double* part = lap_partials(work, nz, ny, nx, is_complex);
  if (is_complex) {
    HT_CHECK_CUDA(lap_ext<float2>(z, work, nz, ny, nx, st));
    k_lap_apply<float2, 1><<<rows, kRegThreads, 0, st>>>(static_cast<const float2*>(work), nz, ny, nx, 0.f,
                                                         nullptr, static_cast<const float2*>(y), part,
                                                         static_cast<const float2*>(y2));
  } else {
    HT_CHECK_CUDA(lap_ext<float>(z, work, nz, ny, nx, st));
    k_lap_apply<float, 1><<<rows, kRegThreads, 0, st>>>(static_cast<const float*>(work), nz, ny, nx, 0.f,
                                                        nullptr, static_cast<const float*>(y), part,
                                                        static_cast<const float*>(y2));
  }
  count_launch();
  k_lap_finish<<<1, 32, 0, st>>>(part, (int)rows, scale, out, y2 ? out2 : nullptr);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_laplacian_energy(const void* u, int nz, int ny, int nx, int is_complex, double scale, void* work,
                                   double* out, void* stream) {
  using namespace ht;
  HT_REQUIRE(u && out, "ht_laplacian_energy: null pointer");
  HT_REG_CHECK("ht_laplacian_energy");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long plane = (long)ny * nx, n = (long)nz * plane;
  const unsigned nb = reg_grid(n);
  double* part = lap_partials(work, nz, ny, nx, is_complex);
  if (is_complex) {
    HT_CHECK_CUDA(lap_ext<float2>(u, work, nz, ny, nx, st));
    k_lap_energy<float2><<<nb, kRegThreads, 0, st>>>(static_cast<const float2*>(work) + plane, n, part);
  } else {
    HT_CHECK_CUDA(lap_ext<float>(u, work, nz, ny, nx, st));
    k_lap_energy<float><<<nb, kRegThreads, 0, st>>>(static_cast<const float*>(work) + plane, n, part);
  }
  count_launch();
  k_lap_finish<<<1, 32, 0, st>>>(part, (int)nb, scale, out, nullptr);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}
