// Padded-grid Fresnel convolution: the surface of the reference's cuFFTDx
// library (conv2d_create / conv2d_run / conv2d_destroy,
// src/holotomocupy/cuda/conv2d.cu:117-159) and its mirror-pad kernels
// (pad_fwd / pad_adj, src/holotomocupy/cuda_kernels.py:78-127).
//
// The propagator itself never builds the padded grid (prop.cu runs it as DCTs
// on the unpadded image); these entry points serve callers that work on the
// padded 2nz x 2n grid directly, as the reference's tests do.
//
// conv: y[b] = IFFT2(FFT2(x[b]) * H), the inverse unnormalised, in three
// passes over [batch, NY, NX]: a row FFT (x -> y), a column pass that runs
// the column FFT, the product with H's column and the inverse column FFT in
// one shared-memory tile, and an inverse row FFT in place.
#include <vector>

#include "common.cuh"
#include "holotomo_b200_internal.h"
#include "lines.cuh"

namespace ht {
namespace {

struct RowIn {
  const float2* p;
  bool valid;
  __device__ __forceinline__ float2 ld(int k) const { return valid ? p[k] : make_float2(0.f, 0.f); }
};
struct RowOut {
  float2* p;
  bool valid;
  __device__ __forceinline__ void st(int k, float2 v) const {
    if (valid) p[k] = v;
  }
};

template <int N, bool INV>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_conv_rows(const float2* in, float2* out, long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < nrows;
  const long r = valid ? row : 0;
  SmRow sm{smem + line * SmRow::padded(N)};
  fft_line_io<N, INV>(RowIn{in + r * N, valid}, sm, RowOut{out + r * N, valid}, t, tw4, line_sync<T>());
}

// data [nimg, N, ncols] in place along the column axis, times H[k, col]
// between the forward and inverse column transforms.
template <int N>
__global__ void __launch_bounds__(ColCfg<N>::THREADS, ColCfg<N>::MIN_BLOCKS)
k_conv_cols(float2* data, int ncols, const float2* __restrict__ H, const float2* __restrict__ tw4) {
  constexpr int C = ColCfg<N>::C;
  constexpr int T = ColCfg<N>::T;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const bool valid = blockIdx.x * C + c < ncols;
  const int col = min((int)blockIdx.x * C + c, ncols - 1);
  float2* img = data + (long)blockIdx.y * N * ncols + col;
  SmCol<C> sm{tile + c};
  fft_line_from<N, false, typename ColCfg<N>::PL>(GColIn{img, ncols, valid}, sm, t, tw4);
  for (int k = t; k < N; k += T) sm.st(k, cmul(sm.ld(k), __ldg(&H[(long)k * ncols + col])));
  __syncthreads();
  fft_line_to<N, true, typename ColCfg<N>::PL>(sm, GColOut{img, ncols, valid}, t, tw4);
}

// Mirror map of the padded grid onto the image along one axis: padded index
// i in [0, 2m) reads image index i - m/2, reflected at both edges (the
// half-sample-symmetric extension of propagation.py:46-56).
__device__ __forceinline__ int mirror_src(int i, int m) {
  const int j = i - m / 2;
  return j < 0 ? -1 - j : (j >= m ? 2 * m - 1 - j : j);
}
// The other padded index that mirror_src maps onto image index j (besides
// j + m/2).
__device__ __forceinline__ int mirror_twin(int j, int m) { return j < m / 2 ? m / 2 - 1 - j : 2 * m + m / 2 - 1 - j; }

// fpad[b, 2nz, 2n] = mirror-padded f[b, nz, n]; one thread per padded sample
__global__ void k_pad_mirror(const float2* __restrict__ f, float2* __restrict__ g, int n, int nz, long total) {
  const long w = 2L * n, h = 2L * nz;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long b = i / (w * h);
    const int Y = (int)((i / w) % h), X = (int)(i % w);
    g[i] = f[(b * nz + mirror_src(Y, nz)) * n + mirror_src(X, n)];
  }
}

// f[b, nz, n] = the adjoint of k_pad_mirror: each image sample sums the four
// padded samples that copy it
__global__ void k_pad_fold(const float2* __restrict__ g, float2* __restrict__ f, int n, int nz, long total) {
  const long w = 2L * n, h = 2L * nz;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const long b = i / ((long)n * nz);
    const int y = (int)((i / n) % nz), x = (int)(i % n);
    const float2* gb = g + b * w * h;
    const long y0 = (long)(y + nz / 2) * w, y1 = (long)mirror_twin(y, nz) * w;
    const int x0 = x + n / 2, x1 = mirror_twin(x, n);
    const float2 a = gb[y0 + x0], bb = gb[y0 + x1], c = gb[y1 + x0], d = gb[y1 + x1];
    f[i] = make_float2((a.x + bb.x) + (c.x + d.x), (a.y + bb.y) + (c.y + d.y));
  }
}

template <int N>
cudaError_t l_conv_rows(bool inv, const float2* in, float2* out, long nrows, const float2* tw, cudaStream_t st) {
  using CF = RowCfg<N>;
  const unsigned grid = (unsigned)((nrows + CF::LINES - 1) / CF::LINES);
  if (inv) {
    cudaError_t e = allow_smem(k_conv_rows<N, true>, CF::SMEM);
    if (e != cudaSuccess) return e;
    k_conv_rows<N, true><<<grid, CF::THREADS, CF::SMEM, st>>>(in, out, nrows, tw);
  } else {
    cudaError_t e = allow_smem(k_conv_rows<N, false>, CF::SMEM);
    if (e != cudaSuccess) return e;
    k_conv_rows<N, false><<<grid, CF::THREADS, CF::SMEM, st>>>(in, out, nrows, tw);
  }
  count_launch();
  return cudaGetLastError();
}

template <int N>
cudaError_t l_conv_cols(float2* data, long nimg, int ncols, const float2* H, const float2* tw, cudaStream_t st) {
  using CF = ColCfg<N>;
  cudaError_t e = allow_smem(k_conv_cols<N>, CF::SMEM);
  if (e != cudaSuccess) return e;
  k_conv_cols<N><<<dim3((ncols + CF::C - 1) / CF::C, (unsigned)nimg), CF::THREADS, CF::SMEM, st>>>(data, ncols, H,
                                                                                                 tw);
  count_launch();
  return cudaGetLastError();
}

cudaError_t conv_rows(int N, bool inv, const float2* in, float2* out, long nrows, const float2* tw, cudaStream_t st) {
  switch (N) {
#define X(S) \
  case S:    \
    return l_conv_rows<S>(inv, in, out, nrows, tw, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t conv_cols(int N, float2* data, long nimg, int ncols, const float2* H, const float2* tw, cudaStream_t st) {
  switch (N) {
#define X(S) \
  case S:    \
    return l_conv_cols<S>(data, nimg, ncols, H, tw, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

unsigned elementwise_grid(long total) {
  const long blocks = (total + 255) / 256;
  return (unsigned)std::min<long>(blocks, 148L * 32);
}

}  // namespace
}  // namespace ht

// ================================================================= C ABI
struct ht_conv2d_s {
  int rows, cols, device;  // image rows (column-transform length), columns
  const float2* tw_x;
  const float2* tw_y;
};

extern "C" int ht_conv2d_create(int rows, int cols, ht_conv2d_s** out) {
  using namespace ht;
  HT_REQUIRE(out != nullptr, "ht_conv2d_create: null pointer");
  if (!fft_size_supported(rows) || !fft_size_supported(cols)) {
    set_error("ht_conv2d_create: rows and cols must be supported FFT lengths (2^a 3^b from 18 to 4096)");
    return kUnsupported;
  }
  int dev = 0;
  HT_CHECK_CUDA(cudaGetDevice(&dev));
  const float2* tx = twiddle_table(cols, dev);
  const float2* ty = twiddle_table(rows, dev);
  if (!tx || !ty) return kCudaError;
  *out = new ht_conv2d_s{rows, cols, dev, tx, ty};
  return kOk;
}

extern "C" int ht_conv2d_destroy(ht_conv2d_s* h) {
  delete h;
  return ht::kOk;
}

extern "C" int ht_conv2d_run(ht_conv2d_s* h, const void* x, const void* H, void* y, long batch, void* stream) {
  using namespace ht;
  HT_REQUIRE(h && x && H && y, "ht_conv2d_run: null pointer");
  HT_REQUIRE(batch >= 0 && batch <= 65535, "ht_conv2d_run: batch must be in [0, 65535]");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float2* yo = static_cast<float2*>(y);
  HT_CHECK_CUDA(conv_rows(h->cols, false, static_cast<const float2*>(x), yo, batch * h->rows, h->tw_x, st));
  HT_CHECK_CUDA(conv_cols(h->rows, yo, batch, h->cols, static_cast<const float2*>(H), h->tw_y, st));
  HT_CHECK_CUDA(conv_rows(h->cols, true, yo, yo, batch * h->rows, h->tw_x, st));
  return kOk;
}

extern "C" int ht_pad_mirror(const void* f, void* fpad, long batch, int nz, int n, void* stream) {
  using namespace ht;
  HT_REQUIRE(f && fpad, "ht_pad_mirror: null pointer");
  HT_REQUIRE(n > 0 && nz > 0 && n % 2 == 0 && nz % 2 == 0 && batch >= 0,
             "ht_pad_mirror: n and nz must be positive and even");
  const long total = batch * 4L * n * nz;
  if (total == 0) return kOk;
  k_pad_mirror<<<elementwise_grid(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(f), static_cast<float2*>(fpad), n, nz, total);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_pad_fold(const void* fpad, void* f, long batch, int nz, int n, void* stream) {
  using namespace ht;
  HT_REQUIRE(f && fpad, "ht_pad_fold: null pointer");
  HT_REQUIRE(n > 0 && nz > 0 && n % 2 == 0 && nz % 2 == 0 && batch >= 0,
             "ht_pad_fold: n and nz must be positive and even");
  const long total = batch * (long)n * nz;
  if (total == 0) return kOk;
  k_pad_fold<<<elementwise_grid(total), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(fpad), static_cast<float2*>(f), n, nz, total);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}
