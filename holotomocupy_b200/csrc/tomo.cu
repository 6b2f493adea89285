// USFFT Radon transform R / RT (reference: src/holotomocupy/tomo.py:12-116,
// gather kernel src/holotomocupy/cuda_kernels.py:3-76).
//
// R(obj)[theta, z, :] = crop . IFFT_n . gather_theta . FFT2_2n . embed(obj * phi)
// with the reference's fftshift-by-sign multiplications folded into the
// passes:
//   1. row pass (length 2n) over the n non-zero rows of each padded slice:
//      embed obj*phi, pre-sign (-1)^(row+col), FFT, post column sign (-1)^kx;
//   2. column pass (length 2n): only rows n/2..3n/2 are non-zero; FFT, post
//      row sign (-1)^ky -> the centred spectrum fde[z] (2n x 2n);
//   3. gather + detector IFFT: for each (theta, z) the n polar samples are
//      81-tap Gaussian-weighted sums of fde[z] (m = 4 at every supported
//      size), then sign, IFFT_n, sign, /4, in one kernel.
// RT runs the exact adjoint: detector FFT with signs; a tiled scatter that
// accumulates each 32x32 tile of fde in shared memory over the polar samples
// whose windows reach it (no global atomics); column IFFT keeping only the
// central rows; row IFFT, crop, * phi.
//
// Angle cosines and sines come from a table computed in double precision on
// the host (the reference's __cosf/__sinf error of ~5e-7 moves R by up to
// ~1e-4 relative at n >= 512, so the exact values are used).
#include "lines.cuh"
#include "holotomo_b200_internal.h"

#include <cmath>
#include <vector>

namespace ht {

struct GatherGeom {
  int n, ntheta, m;
  float coeff0, coeff1;  // pi/mu, -pi^2/mu
  const float2* cs;      // [ntheta] (cos theta, sin theta)
};

// ------------------------------------------------------ pass 1: rows (R)
// obj [nz, n, n] -> fa [nz, n, 2n]
template <int N2>
__global__ void __launch_bounds__(RowCfg<N2>::THREADS)
k_tomo_rows_fwd(const float2* __restrict__ obj, const float* __restrict__ phi, float2* __restrict__ fa,
                long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N2>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N2>::LINES + line;  // z*n + r
  const bool valid = row < nrows;
  SmRow sm{smem + line * SmRow::padded(N2)};
  const int r = valid ? (int)(row % n) : 0;
  const int pr = r + n / 2;
  for (int q = t; q < N2; q += T) {
    float2 v = make_float2(0.f, 0.f);
    if (valid && q >= n / 2 && q < 3 * n / 2) {
      const float2 o = obj[row * n + (q - n / 2)];
      float s = phi[r * n + (q - n / 2)];
      if ((pr + q) & 1) s = -s;
      v = cscale(o, s);
    }
    sm.st(q, v);
  }
  __syncthreads();
  fft_line<N2, false>(sm, t, tw4);
  if (!valid) return;
  for (int k = t; k < N2; k += T) {
    float2 v = sm.ld(k);
    if (k & 1) v = make_float2(-v.x, -v.y);
    fa[row * N2 + k] = v;
  }
}

// --------------------------------------------------- pass 2: columns (R)
// fa [nz, n, 2n] -> fde [nz, 2n, 2n]
template <int N2>
__global__ void __launch_bounds__(ColCfg<N2>::THREADS)
k_tomo_cols_fwd(const float2* __restrict__ fa, float2* __restrict__ fde, const float2* __restrict__ tw4) {
  constexpr int C = ColCfg<N2>::C;
  constexpr int T = ColCfg<N2>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const int col0 = blockIdx.x * C;
  const long z = blockIdx.y;
  const float2* src = fa + z * n * N2;
  for (int idx = threadIdx.x; idx < N2 * C; idx += blockDim.x) {
    const int pr = idx / C, cc = idx % C;
    const bool in = pr >= n / 2 && pr < 3 * n / 2 && col0 + cc < N2;
    tile[idx] = in ? src[(long)(pr - n / 2) * N2 + col0 + cc] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_line<N2, false>(SmCol<C>{tile + c}, t, tw4);
  float2* dst = fde + z * N2 * N2;
  for (int idx = threadIdx.x; idx < N2 * C; idx += blockDim.x) {
    const int ky = idx / C, cc = idx % C;
    if (col0 + cc >= N2) continue;
    float2 v = tile[idx];
    if (ky & 1) v = make_float2(-v.x, -v.y);
    dst[(long)ky * N2 + col0 + cc] = v;
  }
}

// ---------------------------------------------- the 9x9 Gaussian window
// For sample tx of angle th: base indices and separable weights
// (cuda_kernels.py:22-45).  x0 = (tx - n/2)/n cos(th), y0 = -(tx - n/2)/n sin(th).
struct Window {
  int bx, by;
  float ex[9], ey[9];
};

__device__ __forceinline__ void make_window(const GatherGeom& G, int tx, float2 cs, Window& w) {
  const int n = G.n;
  const float twon = (float)(2 * n);
  const float inv_twon = 1.0f / twon;
  const float rho = (float)(tx - n / 2) / (float)n;
  const float x0 = rho * cs.x;
  const float y0 = -rho * cs.y;
  w.bx = (int)floorf(twon * x0) - G.m;
  w.by = (int)floorf(twon * y0) - G.m;
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const float w0 = (float)(w.bx + i) * inv_twon - x0;
    w.ex[i] = __expf(G.coeff1 * w0 * w0);
    const float w1 = (float)(w.by + i) * inv_twon - y0;
    w.ey[i] = G.coeff0 * __expf(G.coeff1 * w1 * w1);
  }
}

// --------------------------------- pass 3: gather + detector IFFT (R)
// fde [nz, 2n, 2n] -> sino [ntheta, nz, n]; one line per (theta, z),
// lines ordered z-major so consecutive CTAs share the same fde slice.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_gather_ifft(const float2* __restrict__ fde, float2* __restrict__ sino, GatherGeom G, int nz,
              const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  constexpr int twon = 2 * N;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long L = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = L < (long)nz * G.ntheta;
  const int z = valid ? (int)(L / G.ntheta) : 0;
  const int th = valid ? (int)(L % G.ntheta) : 0;
  SmRow sm{smem + line * SmRow::padded(N)};
  const float2 cs = G.cs[th];
  const float2* f = fde + (long)z * twon * twon;
  for (int tx = t; tx < N; tx += T) {
    float2 acc = make_float2(0.f, 0.f);
    if (valid) {
      Window w;
      make_window(G, tx, cs, w);
#pragma unroll
      for (int i1 = 0; i1 < 9; ++i1) {
        const int row = (N + w.by + i1 + twon) % twon;
        const float2* frow = f + (long)row * twon;
        float2 ra = make_float2(0.f, 0.f);
#pragma unroll
        for (int i0 = 0; i0 < 9; ++i0) {
          const float2 v = __ldg(&frow[(N + w.bx + i0 + twon) % twon]);
          ra.x += w.ex[i0] * v.x;
          ra.y += w.ex[i0] * v.y;
        }
        acc.x += w.ey[i1] * ra.x;
        acc.y += w.ey[i1] * ra.y;
      }
      // /n of the gather, (-1)^tx sign before the IFFT
      const float s = ((tx & 1) ? -1.f : 1.f) / (float)N;
      acc = cscale(acc, s);
    }
    sm.st(tx, acc);
  }
  __syncthreads();
  fft_line<N, true>(sm, t, tw4);
  if (!valid) return;
  float2* dst = sino + ((long)th * nz + z) * N;
  for (int k = t; k < N; k += T) {
    // ifft 1/n, (-1)^k sign, /4
    const float s = ((k & 1) ? -1.f : 1.f) / (4.f * (float)N);
    dst[k] = cscale(sm.ld(k), s);
  }
}

// --------------------------------------- RT pass 1: detector FFT rows
// sino [ntheta, nz, n] -> G [ntheta, nz, n]:  G = c1d * FFT(c1d * sino)
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_sino_fft(const float2* __restrict__ sino, float2* __restrict__ out, long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < nrows;
  SmRow sm{smem + line * SmRow::padded(N)};
  for (int k = t; k < N; k += T) {
    float2 v = valid ? sino[row * N + k] : make_float2(0.f, 0.f);
    if (k & 1) v = make_float2(-v.x, -v.y);
    sm.st(k, v);
  }
  __syncthreads();
  fft_line<N, false>(sm, t, tw4);
  if (!valid) return;
  for (int k = t; k < N; k += T) {
    float2 v = sm.ld(k);
    if (k & 1) v = make_float2(-v.x, -v.y);
    out[row * N + k] = v;
  }
}

// ----------------------------------------- RT pass 2: tiled scatter
// G [ntheta, nz, n] -> fde [nz, 2n, 2n]; CTA = one TSxTS tile of one slice.
constexpr int kTile = 32;
constexpr int kScatterWarps = 8;

__global__ void __launch_bounds__(kScatterWarps * 32)
k_scatter_tiles(const float2* __restrict__ Gs, float2* __restrict__ fde, GatherGeom G, int nz) {
  __shared__ float2 acc[kTile * kTile];
  const int n = G.n, twon = 2 * n;
  const int X0 = blockIdx.x * kTile, Y0 = blockIdx.y * kTile;
  const int z = blockIdx.z;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) acc[i] = make_float2(0.f, 0.f);
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const float mrg = (float)(G.m + 2);
  for (int th = warp; th < G.ntheta; th += kScatterWarps) {
    const float2 cs = G.cs[th];
    // sample centre in window-base units: cx = 2 rho cos, cy = -2 rho sin, rho = tx - n/2;
    // grid column X = (n + ell) mod 2n.  Check the 3x3 periodic images.
    for (int sy = -1; sy <= 1; ++sy) {
      for (int sx = -1; sx <= 1; ++sx) {
        const float xlo = (float)(X0 - n + sx * twon) - mrg, xhi = (float)(X0 - n + kTile + sx * twon) + mrg;
        const float ylo = (float)(Y0 - n + sy * twon) - mrg, yhi = (float)(Y0 - n + kTile + sy * twon) + mrg;
        float rlo = -(float)(n / 2), rhi = (float)(n / 2);
        const float c2 = 2.f * cs.x, s2 = -2.f * cs.y;
        if (fabsf(c2) > 1e-12f) {
          float a = xlo / c2, b = xhi / c2;
          rlo = fmaxf(rlo, fminf(a, b));
          rhi = fminf(rhi, fmaxf(a, b));
        } else if (xlo > 0.f || xhi < 0.f) {
          continue;
        }
        if (fabsf(s2) > 1e-12f) {
          float a = ylo / s2, b = yhi / s2;
          rlo = fmaxf(rlo, fminf(a, b));
          rhi = fminf(rhi, fmaxf(a, b));
        } else if (ylo > 0.f || yhi < 0.f) {
          continue;
        }
        if (rlo > rhi) continue;
        const int t0 = max(0, (int)floorf(rlo) + n / 2 - 1);
        const int t1 = min(n - 1, (int)ceilf(rhi) + n / 2 + 1);
        for (int tx = t0 + lane; tx <= t1; tx += 32) {
          Window w;
          make_window(G, tx, cs, w);
          const float2 g = Gs[((long)th * nz + z) * n + tx];
#pragma unroll
          for (int i1 = 0; i1 < 9; ++i1) {
            const int row = (n + w.by + i1 + twon) % twon - Y0;
            if (row < 0 || row >= kTile) continue;
#pragma unroll
            for (int i0 = 0; i0 < 9; ++i0) {
              const int col = (n + w.bx + i0 + twon) % twon - X0;
              if (col < 0 || col >= kTile) continue;
              const float wt = w.ex[i0] * w.ey[i1];
              atomicAdd(&acc[row * kTile + col].x, wt * g.x);
              atomicAdd(&acc[row * kTile + col].y, wt * g.y);
            }
          }
        }
      }
    }
  }
  __syncthreads();
  float2* dst = fde + (long)z * twon * twon;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) {
    const int r = i / kTile, c = i % kTile;
    if (Y0 + r < twon && X0 + c < twon) dst[(long)(Y0 + r) * twon + X0 + c] = acc[i];
  }
}

// ------------------------------------------ RT pass 3: column IFFT
// fde [nz, 2n, 2n] -> fb [nz, n, 2n] (central rows only)
template <int N2>
__global__ void __launch_bounds__(ColCfg<N2>::THREADS)
k_tomo_cols_adj(const float2* __restrict__ fde, float2* __restrict__ fb, const float2* __restrict__ tw4) {
  constexpr int C = ColCfg<N2>::C;
  constexpr int T = ColCfg<N2>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const int col0 = blockIdx.x * C;
  const long z = blockIdx.y;
  const float2* src = fde + z * N2 * N2;
  for (int idx = threadIdx.x; idx < N2 * C; idx += blockDim.x) {
    const int ky = idx / C, cc = idx % C;
    float2 v = (col0 + cc < N2) ? src[(long)ky * N2 + col0 + cc] : make_float2(0.f, 0.f);
    if ((ky + col0 + cc) & 1) v = make_float2(-v.x, -v.y);  // pre-sign (-1)^(ky+kx)
    tile[idx] = v;
  }
  __syncthreads();
  fft_line<N2, true>(SmCol<C>{tile + c}, t, tw4);
  float2* dst = fb + z * n * N2;
  const float s = 1.0f / (float)N2;
  for (int idx = threadIdx.x; idx < n * C; idx += blockDim.x) {
    const int r = idx / C, cc = idx % C;
    if (col0 + cc >= N2) continue;
    const int pr = r + n / 2;
    float2 v = cscale(tile[pr * C + cc], (pr & 1) ? -s : s);  // post row sign
    dst[(long)r * N2 + col0 + cc] = v;
  }
}

// --------------------------------------------- RT pass 4: row IFFT
// fb [nz, n, 2n] -> out [nz, n, n] = crop(IFFT) * post column sign * phi
template <int N2>
__global__ void __launch_bounds__(RowCfg<N2>::THREADS)
k_tomo_rows_adj(const float2* __restrict__ fb, const float* __restrict__ phi, float2* __restrict__ out,
                long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N2>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N2>::LINES + line;
  const bool valid = row < nrows;
  SmRow sm{smem + line * SmRow::padded(N2)};
  for (int k = t; k < N2; k += T) sm.st(k, valid ? fb[row * N2 + k] : make_float2(0.f, 0.f));
  __syncthreads();
  fft_line<N2, true>(sm, t, tw4);
  if (!valid) return;
  const int r = (int)(row % n);
  const float s = 1.0f / (float)N2;
  for (int q = t + n / 2; q < 3 * n / 2; q += T) {
    // note: loop covers q in [n/2, 3n/2) with stride T
    float ph = phi[r * n + (q - n / 2)] * s;
    if (q & 1) ph = -ph;
    out[row * n + (q - n / 2)] = cscale(sm.ld(q), ph);
  }
}

// ================================================================ launch
#define HT_LAUNCH_ROWS(K, N, nrows, st, ...)                                                 \
  do {                                                                                        \
    using CF = RowCfg<N>;                                                                     \
    cudaError_t _e = allow_smem(K<N>, CF::SMEM);                                              \
    if (_e != cudaSuccess) return _e;                                                         \
    const long _g = ((nrows) + CF::LINES - 1) / CF::LINES;                                    \
    K<N><<<(unsigned)_g, CF::THREADS, CF::SMEM, st>>>(__VA_ARGS__); ::ht::count_launch();                           \
    return cudaGetLastError();                                                                \
  } while (0)

#define HT_LAUNCH_COLS(K, N, ncols, nimg, st, ...)                                           \
  do {                                                                                        \
    using CF = ColCfg<N>;                                                                     \
    cudaError_t _e = allow_smem(K<N>, CF::SMEM);                                              \
    if (_e != cudaSuccess) return _e;                                                         \
    dim3 _g(((ncols) + CF::C - 1) / CF::C, (unsigned)(nimg));                                 \
    K<N><<<_g, CF::THREADS, CF::SMEM, st>>>(__VA_ARGS__); ::ht::count_launch();                                     \
    return cudaGetLastError();                                                                \
  } while (0)

template <int N2>
static cudaError_t l_rows_fwd(const float2* obj, const float* phi, float2* fa, long nrows, const float2* tw,
                              cudaStream_t st) {
  HT_LAUNCH_ROWS(k_tomo_rows_fwd, N2, nrows, st, obj, phi, fa, nrows, tw);
}
template <int N2>
static cudaError_t l_cols_fwd(const float2* fa, float2* fde, int nz, const float2* tw, cudaStream_t st) {
  HT_LAUNCH_COLS(k_tomo_cols_fwd, N2, N2, nz, st, fa, fde, tw);
}
template <int N>
static cudaError_t l_gather(const float2* fde, float2* sino, const GatherGeom& G, int nz, const float2* tw,
                            cudaStream_t st) {
  HT_LAUNCH_ROWS(k_gather_ifft, N, (long)nz * G.ntheta, st, fde, sino, G, nz, tw);
}
template <int N>
static cudaError_t l_sino_fft(const float2* sino, float2* out, long nrows, const float2* tw, cudaStream_t st) {
  HT_LAUNCH_ROWS(k_sino_fft, N, nrows, st, sino, out, nrows, tw);
}
template <int N2>
static cudaError_t l_cols_adj(const float2* fde, float2* fb, int nz, const float2* tw, cudaStream_t st) {
  HT_LAUNCH_COLS(k_tomo_cols_adj, N2, N2, nz, st, fde, fb, tw);
}
template <int N2>
static cudaError_t l_rows_adj(const float2* fb, const float* phi, float2* out, long nrows, const float2* tw,
                              cudaStream_t st) {
  HT_LAUNCH_ROWS(k_tomo_rows_adj, N2, nrows, st, fb, phi, out, nrows, tw);
}

#define HT_TOMO_SIZES(X) X(18, 36) X(24, 48) X(32, 64) X(48, 96) X(64, 128) X(96, 192) X(128, 256) \
  X(192, 384) X(256, 512) X(384, 768) X(512, 1024) X(768, 1536) X(1024, 2048) X(1536, 3072) X(2048, 4096)

}  // namespace ht

// ================================================================= C ABI
struct ht_tomo_s {
  int n, nz, ntheta, m, device;
  float mu;
  float* phi;          // [n, n] deapodisation * mask * norm (the reference's phi)
  float2* cs;          // [ntheta] (cos, sin) of the angles
  float2* fde;         // workspace [nz, 2n, 2n]
  float2* fab;         // workspace [nz, n, 2n]
  float2* gs;          // workspace [ntheta, nz, n]
  const float2* tw_n;
  const float2* tw_2n;
};

static bool tomo_size_ok(int n) {
  switch (n) {
#define X(A, B) case A:
    HT_TOMO_SIZES(X)
#undef X
    return true;
    default:
      return false;
  }
}

extern "C" int ht_tomo_create(int n, int nz, int ntheta, const float* theta_host, const float* phi_host,
                              ht_tomo_s** out) {
  using namespace ht;
  HT_REQUIRE(out && theta_host && phi_host, "ht_tomo_create: null pointer");
  HT_REQUIRE(n > 0 && nz > 0 && ntheta > 0, "ht_tomo_create: sizes must be positive");
  if (!tomo_size_ok(n)) {
    set_error("ht_tomo_create: n must be one of 18,24,32,48,64,96,128,192,256,384,512,768,1024,1536,2048");
    return kUnsupported;
  }
  // USFFT parameters (tomo.py:14-16)
  const double eps = 1e-3;
  const double mu = -std::log(eps) / (2.0 * n * n);
  const int m = (int)std::ceil(2.0 * n / M_PI * std::sqrt(-mu * std::log(eps) + (mu * n) * (mu * n) / 4.0));
  if (m != 4) {
    set_error("ht_tomo_create: the gridding half-width m must be 4 (it is for every n >= 8)");
    return kUnsupported;
  }
  ht_tomo_s* t = new ht_tomo_s{};
  t->n = n;
  t->nz = nz;
  t->ntheta = ntheta;
  t->m = m;
  t->mu = (float)mu;
  cudaGetDevice(&t->device);
  std::vector<float2> cs(ntheta);
  for (int i = 0; i < ntheta; ++i) {
    const double th = (double)theta_host[i];
    cs[i] = make_float2((float)std::cos(th), (float)std::sin(th));
  }
  t->tw_n = twiddle_table(n, t->device);
  t->tw_2n = twiddle_table(2 * n, t->device);
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
  };
  alloc((void**)&t->phi, sizeof(float) * n * n);
  alloc((void**)&t->cs, sizeof(float2) * ntheta);
  alloc((void**)&t->fde, sizeof(float2) * (size_t)nz * 4 * n * n);
  alloc((void**)&t->fab, sizeof(float2) * (size_t)nz * 2 * n * n);
  alloc((void**)&t->gs, sizeof(float2) * (size_t)ntheta * nz * n);
  if (e == cudaSuccess) e = cudaMemcpy(t->phi, phi_host, sizeof(float) * n * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->cs, cs.data(), sizeof(float2) * ntheta, cudaMemcpyHostToDevice);
  if (e != cudaSuccess || !t->tw_n || !t->tw_2n) {
    if (e != cudaSuccess) set_error(std::string("ht_tomo_create: ") + cudaGetErrorString(e));
    cudaFree(t->phi);
    cudaFree(t->cs);
    cudaFree(t->fde);
    cudaFree(t->fab);
    cudaFree(t->gs);
    delete t;
    return kCudaError;
  }
  *out = t;
  return kOk;
}

extern "C" int ht_tomo_destroy(ht_tomo_s* t) {
  if (!t) return ht::kOk;
  cudaFree(t->phi);
  cudaFree(t->cs);
  cudaFree(t->fde);
  cudaFree(t->fab);
  cudaFree(t->gs);
  delete t;
  return ht::kOk;
}

namespace ht {
static GatherGeom geom(const ht_tomo_s* t) {
  GatherGeom G;
  G.n = t->n;
  G.ntheta = t->ntheta;
  G.m = t->m;
  const float PI = 3.141592653589793238f;
  G.coeff0 = PI / t->mu;
  G.coeff1 = -PI * PI / t->mu;
  G.cs = t->cs;
  return G;
}

static cudaError_t tomo_R_impl(ht_tomo_s* t, const float2* obj, float2* sino, int nz, cudaStream_t st) {
  const GatherGeom G = geom(t);
  cudaError_t e = cudaErrorInvalidValue;
  switch (t->n) {
#define X(A, B)                                                                    \
  case A:                                                                          \
    e = l_rows_fwd<B>(obj, t->phi, t->fab, (long)nz * A, t->tw_2n, st);             \
    if (e == cudaSuccess) e = l_cols_fwd<B>(t->fab, t->fde, nz, t->tw_2n, st);      \
    if (e == cudaSuccess) e = l_gather<A>(t->fde, sino, G, nz, t->tw_n, st);        \
    break;
    HT_TOMO_SIZES(X)
#undef X
    default:
      break;
  }
  return e;
}

static cudaError_t tomo_RT_impl(ht_tomo_s* t, const float2* sino, float2* obj, int nz, cudaStream_t st) {
  const GatherGeom G = geom(t);
  const int n = t->n;
  cudaError_t e = cudaErrorInvalidValue;
  dim3 sgrid((2 * n + kTile - 1) / kTile, (2 * n + kTile - 1) / kTile, nz);
  switch (n) {
#define X(A, B)                                                                          \
  case A:                                                                                \
    e = l_sino_fft<A>(sino, t->gs, (long)t->ntheta * nz, t->tw_n, st);                    \
    if (e == cudaSuccess) {                                                              \
      k_scatter_tiles<<<sgrid, kScatterWarps * 32, 0, st>>>(t->gs, t->fde, G, nz); ::ht::count_launch();        \
      e = cudaGetLastError();                                                            \
    }                                                                                    \
    if (e == cudaSuccess) e = l_cols_adj<B>(t->fde, t->fab, nz, t->tw_2n, st);            \
    if (e == cudaSuccess) e = l_rows_adj<B>(t->fab, t->phi, obj, (long)nz * A, t->tw_2n, st); \
    break;
    HT_TOMO_SIZES(X)
#undef X
    default:
      break;
  }
  return e;
}
}  // namespace ht

extern "C" int ht_tomo_R(ht_tomo_s* t, const void* obj, void* sino, int nz, void* stream) {
  using namespace ht;
  HT_REQUIRE(t && obj && sino, "ht_tomo_R: null pointer");
  HT_REQUIRE(nz >= 0 && nz <= t->nz, "ht_tomo_R: nz exceeds the handle's slice capacity");
  if (nz == 0) return kOk;
  HT_CHECK_CUDA(tomo_R_impl(t, static_cast<const float2*>(obj), static_cast<float2*>(sino), nz,
                            static_cast<cudaStream_t>(stream)));
  return kOk;
}

extern "C" int ht_tomo_RT(ht_tomo_s* t, const void* sino, void* obj, int nz, void* stream) {
  using namespace ht;
  HT_REQUIRE(t && obj && sino, "ht_tomo_RT: null pointer");
  HT_REQUIRE(nz >= 0 && nz <= t->nz, "ht_tomo_RT: nz exceeds the handle's slice capacity");
  if (nz == 0) return kOk;
  HT_CHECK_CUDA(tomo_RT_impl(t, static_cast<const float2*>(sino), static_cast<float2*>(obj), nz,
                             static_cast<cudaStream_t>(stream)));
  return kOk;
}
