// USFFT Radon transform R / RT (reference: src/holotomocupy/tomo.py:12-116,
// gather kernel src/holotomocupy/cuda_kernels.py:3-76).
//
// R(obj)[theta, z, :] = crop . IFFT_n . gather_theta . FFT2_2n . embed(obj * phi)
// with the reference's fftshift-by-sign multiplications folded into the
// passes.  Slices are processed Z at a time in "Z-interleaved" layouts (the Z
// samples of consecutive slices stored together), so every spectral access
// is one Z*8-byte vector and each Gaussian window serves Z slices:
//   1. row pass (length 2n) over the n non-zero rows of the padded slice:
//      embed obj*phi, pre-sign (-1)^(row+col), FFT, post column sign (-1)^kx
//      -> fa  [zb][n][2n][Z];
//   2. column pass (length 2n, rows outside n/2..3n/2 are zero): FFT, post
//      row sign (-1)^ky -> the centred spectrum fde [zb][2n][2n][Z];
//   3. gather + detector IFFT: for each (theta, slice batch) the n polar
//      samples are 81-tap Gaussian-weighted sums of fde (m = 4 at every
//      supported size), then sign, IFFT_n, sign, /4.
// RT runs the exact adjoint: detector FFT with signs -> gs [zb][theta][n][Z];
// a gather replaces the reference's atomic scatter: every
// warp owns an 8 x 4 tile of cells and visits, uniformly across its lanes,
// only the angles whose line passes near the tile (binary search in the
// sorted angles) and the samples whose window can meet it; membership and
// weights come from the forward's own formulas, so R^T is the exact
// transpose of R and deterministic; then column IFFT keeping the central
// rows, row IFFT, crop, * phi.
//
// Angle cosines and sines come from a table computed in double precision on
// the host (the reference's __cosf/__sinf error of ~5e-7 moves R by up to
// ~1e-4 relative at n >= 512, so the exact values are used).
#include "lines.cuh"
#include "holotomo_b200_internal.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

namespace ht {

struct GatherGeom {
  int n, ntheta, m;
  float coeff0, coeff1;   // pi/mu, -pi^2/mu
  const float2* cs;       // [ntheta] (cos theta, sin theta)
  const float* th_sorted; // [ntheta] theta mod pi, ascending
  const int* th_index;    // [ntheta] original index of th_sorted[i]
};

// Slices per batch for padded size N2 = 2n.
template <int N2>
struct TZ {
  static constexpr int Z = (N2 <= 1024) ? 8 : ((N2 == 2048) ? 4 : 2);
};

// Plan of the Radon transform's lines of N samples, Z a CTA: the row plan,
// except that 24 samples a thread are faster for the 384-sample lines and for
// the 768-sample grid lines at n = 384 (Z = 8; BH iteration at 384^3 x 672 x
// 4: 67.5 against 69.0 ms), while the 768-sample detector lines at n = 768
// (Z = 2) keep the 12-sample row plan (R there: 11.6 against 15.1 ms).
template <int N, int Z>
struct RadonPlan : Plan<N> {};
template <int Z>
struct RadonPlan<384, Z> : PlanOf<384, 24, 8, 8, 3, 2> {};
template <>
struct RadonPlan<768, 8> : PlanOf<768, 24, 8, 8, 4, 3> {};

// Z lines of length N per CTA; line stride odd in float2 units so that
// reading one position of all lines is bank-conflict free.
template <int N, int Z>
struct ZCfg {
  using PL = RadonPlan<N, Z>;
  static constexpr int T = PL::T;
  static constexpr int THREADS = Z * T;
  static constexpr int LS = SmRow::padded(N) + 1;
  static constexpr int SMEM = Z * LS * (int)sizeof(float2);
  // lines of whole warps synchronise on named barriers 1..15 (LineSync)
  static_assert(T % 32 != 0 || Z <= 15, "at most 15 line barriers per block");
};

template <int N, int Z>
__device__ __forceinline__ SmRow zline(float2* smem, int l) {
  return SmRow{smem + l * ZCfg<N, Z>::LS};
}

// ---------------------------------------------- the 9x9 Gaussian window
// For sample tx of angle th: base indices and separable weights
// (cuda_kernels.py:22-45).  x0 = (tx - n/2)/n cos(th), y0 = -(tx - n/2)/n sin(th).
struct Window {
  int bx, by;
  float x0, y0;
};

__device__ __forceinline__ void window_base(const GatherGeom& G, int tx, float2 cs, Window& w) {
  const int n = G.n;
  const float twon = (float)(2 * n);
  const float rho = (float)(tx - n / 2) / (float)n;
  w.x0 = rho * cs.x;
  w.y0 = -rho * cs.y;
  w.bx = (int)floorf(twon * w.x0) - G.m;
  w.by = (int)floorf(twon * w.y0) - G.m;
}
__device__ __forceinline__ float wx_tap(const GatherGeom& G, const Window& w, int i) {
  const float inv_twon = 1.0f / (float)(2 * G.n);
  const float w0 = (float)(w.bx + i) * inv_twon - w.x0;
  return __expf(G.coeff1 * w0 * w0);
}
__device__ __forceinline__ float wy_tap(const GatherGeom& G, const Window& w, int i) {
  const float inv_twon = 1.0f / (float)(2 * G.n);
  const float w1 = (float)(w.by + i) * inv_twon - w.y0;
  return G.coeff0 * __expf(G.coeff1 * w1 * w1);
}

// ------------------------------------------------------ 1: rows (R)
// obj [nz, n, n] -> fa [zb][n][2n][Z];  grid (n, nzb)
template <int N2>
__global__ void __launch_bounds__(ZCfg<N2, TZ<N2>::Z>::THREADS)
k_trow_fwd(const float2* __restrict__ obj, const float* __restrict__ phi, float2* __restrict__ fa, int nz,
           const float2* __restrict__ tw4) {
  constexpr int Z = TZ<N2>::Z;
  constexpr int T = ZCfg<N2, Z>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int l = threadIdx.x / T, t = threadIdx.x % T;
  const int r = blockIdx.x, zb = blockIdx.y;
  const int z = zb * Z + l;
  const bool valid = z < nz;
  const int pr = r + n / 2;
  SmRow sm = zline<N2, Z>(smem, l);
  for (int q = t; q < N2; q += T) {
    float2 v = make_float2(0.f, 0.f);
    if (valid && q >= n / 2 && q < 3 * n / 2) {
      float s = phi[r * n + (q - n / 2)];
      if ((pr + q) & 1) s = -s;
      v = cscale(obj[((long)z * n + r) * n + (q - n / 2)], s);
    }
    sm.st(q, v);
  }
  __syncthreads();
  fft_line<N2, false, typename ZCfg<N2, Z>::PL>(sm, t, tw4, line_sync<T>());
  __syncthreads();  // the stores below read every line
  float2* dst = fa + ((long)zb * n + r) * N2 * Z;
  for (int idx = threadIdx.x; idx < N2 * Z; idx += blockDim.x) {
    const int kx = idx / Z, ll = idx % Z;
    float2 v = zline<N2, Z>(smem, ll).ld(kx);
    if (kx & 1) v = make_float2(-v.x, -v.y);
    dst[idx] = v;
  }
}

// --------------------------------------------------- 2: columns (R)
// fa [zb][n][2n][Z] -> fde [zb][2n][2n][Z];  grid (2n, nzb).  Thread
// (t, l = threadIdx.x % Z) works on slice l, so a warp reads and writes whole
// Z-vectors of 32 / Z rows; the first FFT stage loads from fa (zero outside
// the central n rows) and the last stores to fde (with the (-1)^ky sign), so
// the column passes shared memory only between stages.
template <int Z>
struct TColFwdIn {
  const float2* p;  // fa at row 0 of this column and slice
  int n, rowstride;
  __device__ __forceinline__ float2 ld(int k) const {
    return (k >= n / 2 && k < 3 * n / 2) ? p[(long)(k - n / 2) * rowstride] : make_float2(0.f, 0.f);
  }
};
struct TColFwdOut {
  float2* p;  // fde at row 0 of this column and slice
  int rowstride;
  __device__ __forceinline__ void st(int k, float2 v) const {
    p[(long)k * rowstride] = (k & 1) ? make_float2(-v.x, -v.y) : v;
  }
};

template <int N2>
__global__ void __launch_bounds__(ZCfg<N2, TZ<N2>::Z>::THREADS)
k_tcol_fwd(const float2* __restrict__ fa, float2* __restrict__ fde, const float2* __restrict__ tw4) {
  constexpr int Z = TZ<N2>::Z;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int l = threadIdx.x % Z, t = threadIdx.x / Z;
  const int kx = blockIdx.x, zb = blockIdx.y;
  const float2* src = fa + (long)zb * n * N2 * Z + (long)kx * Z + l;
  float2* dst = fde + (long)zb * N2 * N2 * Z + (long)kx * Z + l;
  fft_line_io<N2, false, typename ZCfg<N2, Z>::PL>(TColFwdIn<Z>{src, n, N2 * Z}, SmCol<Z>{smem + l},
                                                   TColFwdOut{dst, N2 * Z}, t, tw4);
}

// ------------------------------------- 3: gather + detector IFFT (R)
// fde [zb][2n][2n][Z] -> sino [ntheta, nz, n];  grid (ntheta, nzb)
// Z/2 consecutive lanes share one polar sample, each lane reading one float4
// (two slices) of every tap's Z-vector, so the lanes of a warp read whole
// 64-byte cell vectors instead of 16 bytes from 32 different cells.
// Register cap of the gather: 64 at 512 threads (two blocks per SM), else 96.
template <int THREADS>
constexpr int gather_max_regs() {
  return THREADS >= 512 ? 64 : 96;
}

template <int N, int THREADS = ZCfg<N, TZ<2 * N>::Z>::THREADS>
__global__ void __maxnreg__(gather_max_regs<THREADS>())
k_tgather(const float2* __restrict__ fde, float2* __restrict__ sino, GatherGeom G, int nz, int ldz,
          const float2* __restrict__ tw4, const float* __restrict__ symx) {
  constexpr int Z = TZ<2 * N>::Z;
  constexpr int Q = Z / 2;                       // lanes per sample
  constexpr int T = ZCfg<N, Z>::T;
  constexpr int twon = 2 * N;
  extern __shared__ float2 smem[];
  const int th = blockIdx.x, zb = blockIdx.y;
  const float2 cs = G.cs[th];
  const int q = threadIdx.x % Q;
  const float4* f = reinterpret_cast<const float4*>(fde + (long)zb * twon * twon * Z) + q;
  for (int tx = threadIdx.x / Q; tx < N; tx += blockDim.x / Q) {
    Window w;
    window_base(G, tx, cs, w);
    float ex[9];
    int cols[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      ex[i] = wx_tap(G, w, i);
      cols[i] = (N + w.bx + i + twon) % twon;
    }
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int i1 = 0; i1 < 9; ++i1) {
      const int row = (N + w.by + i1 + twon) % twon;
      const float ey = wy_tap(G, w, i1);
      const float4* frow = f + (long)row * twon * Q;
      float4 ra = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int i0 = 0; i0 < 9; ++i0) {
        const float4 v = __ldg(&frow[(long)cols[i0] * Q]);
        ra.x += ex[i0] * v.x;
        ra.y += ex[i0] * v.y;
        ra.z += ex[i0] * v.z;
        ra.w += ex[i0] * v.w;
      }
      acc.x += ey * ra.x;
      acc.y += ey * ra.y;
      acc.z += ey * ra.z;
      acc.w += ey * ra.w;
    }
    // /n of the gather, (-1)^tx before the IFFT; symx: the detector-axis
    // filter, whose frequency kx sits at tx = kx - n/2 (mod n) here
    float s = ((tx & 1) ? -1.f : 1.f) / (float)N;
    if (symx) s *= __ldg(&symx[(tx + N / 2) % N]);
    zline<N, Z>(smem, 2 * q).st(tx, make_float2(s * acc.x, s * acc.y));
    zline<N, Z>(smem, 2 * q + 1).st(tx, make_float2(s * acc.z, s * acc.w));
  }
  __syncthreads();
  const int l = threadIdx.x / T, t = threadIdx.x % T;
  fft_line<N, true, typename ZCfg<N, Z>::PL>(zline<N, Z>(smem, l), t, tw4, line_sync<T>());
  const int z = zb * Z + l;
  if (z >= nz) return;
  float2* dst = sino + ((long)th * ldz + z) * N;  // ldz: rows per angle of the sinogram
  SmRow sm = zline<N, Z>(smem, l);
  for (int k = t; k < N; k += T) {
    const float s = ((k & 1) ? -1.f : 1.f) / (4.f * (float)N);  // ifft 1/n, (-1)^k, /4
    dst[k] = cscale(sm.ld(k), s);
  }
}

// ------------------------------------- RT 1: detector FFT with signs
// sino [ntheta, nz, n] -> gs [zb][ntheta][n][Z];  grid (ntheta, nzb)
template <int N>
__global__ void __launch_bounds__(ZCfg<N, TZ<2 * N>::Z>::THREADS)
k_tsino_fft(const float2* __restrict__ sino, float2* __restrict__ gs, int ntheta, int nz, int ldz,
            const float2* __restrict__ tw4, const float* __restrict__ symx, float scale) {
  constexpr int Z = TZ<2 * N>::Z;
  constexpr int T = ZCfg<N, Z>::T;
  extern __shared__ float2 smem[];
  const int l = threadIdx.x / T, t = threadIdx.x % T;
  const int th = blockIdx.x, zb = blockIdx.y;
  const int z = zb * Z + l;
  SmRow sm = zline<N, Z>(smem, l);
  for (int k = t; k < N; k += T) {
    float2 v = (z < nz) ? sino[((long)th * ldz + z) * N + k] : make_float2(0.f, 0.f);
    if (k & 1) v = make_float2(-v.x, -v.y);
    sm.st(k, v);
  }
  __syncthreads();
  fft_line<N, false, typename ZCfg<N, Z>::PL>(sm, t, tw4, line_sync<T>());
  __syncthreads();  // the stores below read every line
  float2* dst = gs + ((long)zb * ntheta + th) * N * Z;
  for (int idx = threadIdx.x; idx < N * Z; idx += blockDim.x) {
    const int tx = idx / Z, ll = idx % Z;
    float2 v = zline<N, Z>(smem, ll).ld(tx);
    float sg = (tx & 1) ? -scale : scale;  // the caller's scale folded into the sign
    if (symx) sg *= __ldg(&symx[(tx + N / 2) % N]);  // detector-axis filter (see k_tgather)
    dst[idx] = cscale(v, sg);
  }
}

// -------------------------------------------- RT 2: sparse cell gather
// The pairs (sample, spectral cell) of R's gridding and their weights depend
// only on the angles, so ht_tomo_create lists them once per cell -- found by
// a per-cell search (the angles whose line passes within 7.5 cells, by binary
// search in the sorted angles; the radial samples near the cell; window
// membership and weights from the forward's own formulas) -- in a sliced
// ELLPACK layout: a small tile of CPS = 64/Z cells forms a slice, entry p of
// the slice is CPS consecutive (sample, weight) pairs, shorter lists padded
// with weight 0.  R^T runs one slice per warp with Z/2 lanes per cell, each
// lane reading one float4 (two slices) of the sample's Z-vector, so a warp
// load covers CPS whole 64-byte vectors; neighbouring cells share samples,
// which L1 serves.  The exact transpose of R, deterministic, no atomics.
constexpr float kLineReach = 7.5f;  // window cells lie within 5 sqrt(2) of the sample centre

__device__ __forceinline__ int lower_bound_f(const float* a, int n, float v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Visit (sample index j*n + t, weight) for every sample of angle j whose window holds cell (X, Y).
template <class F>
__device__ __forceinline__ void cell_angle_pairs(const GatherGeom& G, int j, float px, float py, int X, int Y, F& f) {
  const int n = G.n, twon = 2 * n;
  const float2 cs = G.cs[j];
  const float s = px * cs.x - py * cs.y;  // projection onto (cos, -sin)
  const int t0 = max(0, (int)ceilf((s - kLineReach) * 0.5f) + n / 2);
  const int t1 = min(n - 1, (int)floorf((s + kLineReach) * 0.5f) + n / 2);
  for (int tx = t0; tx <= t1; ++tx) {
    Window w;
    window_base(G, tx, cs, w);
    // (X - n - bx) mod 2n: bx lies in [-n - m, n - m] and X - n in [-n, n), so
    // one correction either way reduces it
    int i0 = X - n - w.bx;
    i0 += (i0 < 0) ? twon : 0;
    i0 -= (i0 >= twon) ? twon : 0;
    if (i0 > 8) continue;
    int i1 = Y - n - w.by;
    i1 += (i1 < 0) ? twon : 0;
    i1 -= (i1 >= twon) ? twon : 0;
    if (i1 > 8) continue;
    f(j * n + tx, wx_tap(G, w, i0) * wy_tap(G, w, i1));
  }
}

// All pairs of cell (X, Y), in a fixed order.
template <class F>
__device__ void cell_pairs(const GatherGeom& G, int X, int Y, F& f) {
  const int n = G.n, twon = 2 * n;
  const float PI = 3.14159265358979f;
  const float lim = (float)n + 9.0f;
  for (int oy = -1; oy <= 1; ++oy) {
    for (int ox = -1; ox <= 1; ++ox) {
      // the cell and its periodic images within reach of the sample disc
      const float px = (float)(X - n + ox * twon), py = (float)(Y - n + oy * twon);
      if (fabsf(px) > lim || fabsf(py) > lim) continue;
      const float R = sqrtf(px * px + py * py);
      if (R <= kLineReach) {
        for (int j = 0; j < G.ntheta; ++j) cell_angle_pairs(G, j, px, py, X, Y, f);
        continue;
      }
      // angles with R |sin(theta + phi)| <= reach, theta taken mod pi
      const float dlt = asinf(fminf(1.0f, kLineReach / R)) + 1e-4f;
      float c = -atan2f(py, px);
      c = c - PI * floorf(c / PI);
      const float a = c - dlt, b = c + dlt;
      float ia[2], ib[2];
      int ni = 0;
      if (a < 0.f) {
        ia[ni] = 0.f;
        ib[ni++] = b;
        ia[ni] = a + PI;
        ib[ni++] = PI;
      } else if (b >= PI) {
        ia[ni] = a;
        ib[ni++] = PI;
        ia[ni] = 0.f;
        ib[ni++] = b - PI;
      } else {
        ia[ni] = a;
        ib[ni++] = b;
      }
      for (int q = 0; q < ni; ++q)
        for (int i = lower_bound_f(G.th_sorted, G.ntheta, ia[q]); i < G.ntheta && G.th_sorted[i] <= ib[q]; ++i)
          cell_angle_pairs(G, G.th_index[i], px, py, X, Y, f);
    }
  }
}

struct PairCount {
  int n = 0;
  __device__ void operator()(int, float) { ++n; }
};

// Slices: tiles of TW x TH = CPS cells (CPS = 64 / Z: 8, 16 or 32 cells).
struct SliceShape {
  int tw, th;
};
__host__ __device__ __forceinline__ SliceShape slice_shape(int cps) {
  return cps == 8 ? SliceShape{4, 2} : (cps == 16 ? SliceShape{4, 4} : SliceShape{8, 4});
}
// slice s, cell k of the slice <-> cell (X, Y) (false: outside the grid)
__device__ __forceinline__ bool slice_cell(long s, int k, int twon, SliceShape sh, int& X, int& Y) {
  const long tiles_x = (twon + sh.tw - 1) / sh.tw;
  X = (int)(s % tiles_x) * sh.tw + k % sh.tw;
  Y = (int)(s / tiles_x) * sh.th + k / sh.tw;
  return X < twon && Y < twon;
}
__device__ __forceinline__ void cell_slice(int X, int Y, int twon, SliceShape sh, long& s, int& k) {
  s = (long)(Y / sh.th) * ((twon + sh.tw - 1) / sh.tw) + X / sh.tw;
  k = (Y % sh.th) * sh.tw + X % sh.tw;
}

// pairs per cell;  cells c = Y * 2n + X
__global__ void k_cell_count(GatherGeom G, int* __restrict__ cnt) {
  const int twon = 2 * G.n;
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long)twon * twon) return;
  PairCount f;
  cell_pairs(G, (int)(c % twon), (int)(c / twon), f);
  cnt[c] = f.n;
}

// slice length = the longest list of its cells
__global__ void k_slice_len(const int* __restrict__ cnt, int twon, int cps, int* __restrict__ len, long nslices) {
  const long s = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslices) return;
  const SliceShape sh = slice_shape(cps);
  int mx = 0;
  for (int k = 0; k < cps; ++k) {
    int X, Y;
    if (slice_cell(s, k, twon, sh, X, Y)) mx = max(mx, cnt[(long)Y * twon + X]);
  }
  len[s] = mx;
}

struct PairFillS {
  int2* dst;  // this cell's first entry; entries cps apart
  int cps;
  int p = 0;
  __device__ void operator()(int idx, float w) {
    dst[(long)p * cps] = make_int2(idx, __float_as_int(w));
    ++p;
  }
};

__global__ void k_cell_fill(GatherGeom G, int cps, const long* __restrict__ off, int2* __restrict__ ent) {
  const int twon = 2 * G.n;
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= (long)twon * twon) return;
  const int X = (int)(c % twon), Y = (int)(c / twon);
  long sl;
  int k;
  cell_slice(X, Y, twon, slice_shape(cps), sl, k);
  PairFillS f{ent + off[sl] * cps + k, cps};
  cell_pairs(G, X, Y, f);
}

// gs [zb][ntheta][n][Z] -> fde [zb][2n][2n][Z]; grid ceil(slices * 32 / 256) * ceil(nzb / ZG)
// blocks (see the block order below); ZG slice batches per lane
template <int Z, int ZG>
__global__ void __launch_bounds__(256)
k_tcell(const float2* __restrict__ gs, float2* __restrict__ fde, const int* __restrict__ len,
        const long* __restrict__ off, const int2* __restrict__ ent, int twon, long nslices, long nsamp, int nzb,
        int ngroups) {
  constexpr int Q = Z / 2;       // lanes per cell
  constexpr int CPS = 32 / Q;    // cells per slice (warp)
  // block b handles the cells of block b / ngroups for the slice batches of
  // group b % ngroups: the ngroups consecutive blocks that read one stretch of
  // the pair lists run together, so the lists come from DRAM once and from L2
  // for the other groups
  const int grp = (int)(blockIdx.x % ngroups);
  const long tid = (long)(blockIdx.x / ngroups) * blockDim.x + threadIdx.x;
  const long sl = tid / 32;
  if (sl >= nslices) return;
  const int lane = (int)(tid % 32), k = lane / Q, q = lane % Q;
  int X, Y;
  const bool live = slice_cell(sl, k, twon, slice_shape(CPS), X, Y);
  const int zb0 = grp * ZG;
  const int nl = len[sl];
  const int2* e = ent + off[sl] * CPS + k;
  float4 acc[ZG];
#pragma unroll
  for (int g = 0; g < ZG; ++g) acc[g] = make_float4(0.f, 0.f, 0.f, 0.f);
  const float4* gb = reinterpret_cast<const float4*>(gs + (long)zb0 * nsamp * Z) + q;
  for (int p = 0; p < nl; ++p) {
    const int2 v = __ldg(&e[(long)p * CPS]);
    const float w = __int_as_float(v.y);
#pragma unroll
    for (int g = 0; g < ZG; ++g)
      if (zb0 + g < nzb) {
        const float4 u = __ldg(&gb[((long)g * nsamp + v.x) * Q]);
        acc[g].x += w * u.x;
        acc[g].y += w * u.y;
        acc[g].z += w * u.z;
        acc[g].w += w * u.w;
      }
  }
  if (!live) return;
  const long c = (long)Y * twon + X, ncells = (long)twon * twon;
#pragma unroll
  for (int g = 0; g < ZG; ++g) {
    if (zb0 + g >= nzb) break;
    reinterpret_cast<float4*>(fde + ((long)(zb0 + g) * ncells + c) * Z)[q] = acc[g];
  }
}

// ------------------------------------------- RT 3: column IFFT
// fde [zb][2n][2n][Z] -> fb [zb][n][2n][Z] (central rows);  grid (2n, nzb).
// Thread layout and direct global first/last stages as in k_tcol_fwd.
struct TColAdjIn {
  const float2* p;  // fde at row 0 of this column and slice
  int rowstride, kx;
  __device__ __forceinline__ float2 ld(int k) const {
    const float2 v = p[(long)k * rowstride];
    return ((k + kx) & 1) ? make_float2(-v.x, -v.y) : v;  // pre-sign (-1)^(ky+kx)
  }
};
struct TColAdjOut {
  float2* p;  // fb at row 0 of this column and slice
  int n, rowstride;
  float s;    // 1 / 2n
  __device__ __forceinline__ void st(int k, float2 v) const {
    if (k >= n / 2 && k < 3 * n / 2) p[(long)(k - n / 2) * rowstride] = cscale(v, (k & 1) ? -s : s);  // post sign
  }
};

template <int N2>
__global__ void __launch_bounds__(ZCfg<N2, TZ<N2>::Z>::THREADS)
k_tcol_adj(const float2* __restrict__ fde, float2* __restrict__ fb, const float2* __restrict__ tw4) {
  constexpr int Z = TZ<N2>::Z;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int l = threadIdx.x % Z, t = threadIdx.x / Z;
  const int kx = blockIdx.x, zb = blockIdx.y;
  const float2* src = fde + (long)zb * N2 * N2 * Z + (long)kx * Z + l;
  float2* dst = fb + (long)zb * n * N2 * Z + (long)kx * Z + l;
  fft_line_io<N2, true, typename ZCfg<N2, Z>::PL>(TColAdjIn{src, N2 * Z, kx}, SmCol<Z>{smem + l},
                                                  TColAdjOut{dst, n, N2 * Z, 1.0f / (float)N2}, t, tw4);
}

// ---------------------------------------------- RT 4: row IFFT
// fb [zb][n][2n][Z] -> out [nz, n, n] = crop(IFFT) * (-1)^q * phi;  grid (n, nzb)
template <int N2>
__global__ void __launch_bounds__(ZCfg<N2, TZ<N2>::Z>::THREADS)
k_trow_adj(const float2* __restrict__ fb, const float* __restrict__ phi, float2* __restrict__ out, int nz,
           const float2* __restrict__ tw4) {
  constexpr int Z = TZ<N2>::Z;
  constexpr int T = ZCfg<N2, Z>::T;
  constexpr int n = N2 / 2;
  extern __shared__ float2 smem[];
  const int l = threadIdx.x / T, t = threadIdx.x % T;
  const int r = blockIdx.x, zb = blockIdx.y;
  const float2* src = fb + ((long)zb * n + r) * N2 * Z;
  for (int idx = threadIdx.x; idx < N2 * Z; idx += blockDim.x) {
    const int kx = idx / Z, ll = idx % Z;
    zline<N2, Z>(smem, ll).st(kx, src[idx]);
  }
  __syncthreads();
  SmRow sm = zline<N2, Z>(smem, l);
  fft_line<N2, true, typename ZCfg<N2, Z>::PL>(sm, t, tw4, line_sync<T>());
  const int z = zb * Z + l;
  if (z >= nz) return;
  const float s = 1.0f / (float)N2;
  for (int q = t + n / 2; q < 3 * n / 2; q += T) {
    float ph = phi[r * n + (q - n / 2)] * s;
    if (q & 1) ph = -ph;
    out[((long)z * n + r) * n + (q - n / 2)] = cscale(sm.ld(q), ph);
  }
}

// ================================================================ launch
template <int N2>
static cudaError_t tomo_R_sized(const float2* obj, float2* sino, const float* phi, float2* fa, float2* fde,
                                const GatherGeom& G, int nz, int ldz, const float2* tw_n, const float2* tw_2n,
                                const float* symx, cudaStream_t st) {
  constexpr int n = N2 / 2;
  constexpr int Z = TZ<N2>::Z;
  using C2 = ZCfg<N2, Z>;
  using C1 = ZCfg<n, Z>;
  const int nzb = (nz + Z - 1) / Z;
  cudaError_t e;
  if ((e = allow_smem(k_trow_fwd<N2>, C2::SMEM)) != cudaSuccess) return e;
  if ((e = allow_smem(k_tcol_fwd<N2>, C2::SMEM)) != cudaSuccess) return e;
  if ((e = allow_smem(k_tgather<n>, C1::SMEM)) != cudaSuccess) return e;
  k_trow_fwd<N2><<<dim3(n, nzb), C2::THREADS, C2::SMEM, st>>>(obj, phi, fa, nz, tw_2n);
  count_launch();
  k_tcol_fwd<N2><<<dim3(N2, nzb), C2::THREADS, C2::SMEM, st>>>(fa, fde, tw_2n);
  count_launch();
  {
    KTimer kt("k_tgather", st, (double)nz);
    k_tgather<n><<<dim3(G.ntheta, nzb), C1::THREADS, C1::SMEM, st>>>(fde, sino, G, nz, ldz, tw_n, symx);
  }
  count_launch();
  return cudaGetLastError();
}

struct CellLists {
  const int* len;   // [nslices]
  const long* off;  // [nslices] first entry of each slice (in entries of 32)
  const int2* ent;  // entries
};

template <int N2>
static cudaError_t tomo_RT_sized(const float2* sino, float2* obj, const float* phi, float2* fab, float2* fde,
                                 float2* gs, const GatherGeom& G, const CellLists& L, int nz, int ldz,
                                 const float2* tw_n,
                                 const float2* tw_2n, const float* symx, float scale, cudaStream_t st) {
  constexpr int n = N2 / 2;
  constexpr int Z = TZ<N2>::Z;
  using C2 = ZCfg<N2, Z>;
  using C1 = ZCfg<n, Z>;
  const int nzb = (nz + Z - 1) / Z;
  cudaError_t e;
  if ((e = allow_smem(k_tsino_fft<n>, C1::SMEM)) != cudaSuccess) return e;
  if ((e = allow_smem(k_tcol_adj<N2>, C2::SMEM)) != cudaSuccess) return e;
  if ((e = allow_smem(k_trow_adj<N2>, C2::SMEM)) != cudaSuccess) return e;
  k_tsino_fft<n><<<dim3(G.ntheta, nzb), C1::THREADS, C1::SMEM, st>>>(sino, gs, G.ntheta, nz, ldz, tw_n, symx,
                                                                    scale);
  count_launch();
  {
    KTimer kt("k_tcell", st, (double)nz);
    constexpr int ZG = 2;  // slice batches per read of the pair lists
    const SliceShape sh = slice_shape(64 / Z);
    const long nsl = (long)((N2 + sh.tw - 1) / sh.tw) * ((N2 + sh.th - 1) / sh.th);
    const int ngroups = (nzb + ZG - 1) / ZG;
    const long nblk = (nsl * 32 + 255) / 256;
    k_tcell<Z, ZG><<<(unsigned)(nblk * ngroups), 256, 0, st>>>(gs, fde, L.len, L.off, L.ent, N2, nsl,
                                                            (long)G.ntheta * n, nzb, ngroups);
  }
  count_launch();
  k_tcol_adj<N2><<<dim3(N2, nzb), C2::THREADS, C2::SMEM, st>>>(fde, fab, tw_2n);
  count_launch();
  k_trow_adj<N2><<<dim3(n, nzb), C2::THREADS, C2::SMEM, st>>>(fab, phi, obj, nz, tw_2n);
  count_launch();
  return cudaGetLastError();
}

#define HT_TOMO_SIZES(X) X(18, 36) X(24, 48) X(32, 64) X(48, 96) X(64, 128) X(96, 192) X(128, 256) \
  X(192, 384) X(256, 512) X(384, 768) X(512, 1024) X(768, 1536) X(1024, 2048) X(1536, 3072) X(2048, 4096)

static int tomo_Z(int n) {
  const int N2 = 2 * n;
  return (N2 <= 1024) ? 8 : ((N2 == 2048) ? 4 : 2);
}

}  // namespace ht

// ================================================================= C ABI
struct ht_tomo_s {
  int n, nz, ntheta, m, device;
  float mu;
  float* phi;          // [n, n] deapodisation * mask * norm (the reference's phi)
  float2* cs;          // [ntheta] (cos, sin) of the angles
  float* th_sorted;    // [ntheta] angles mod pi, ascending
  int* th_index;       // [ntheta]
  float2* fde;         // workspace [nzb][2n][2n][Z]
  float2* fab;         // workspace [nzb][n][2n][Z]
  float2* gs;          // workspace [nzb][ntheta][n][Z]
  const float2* tw_n;
  const float2* tw_2n;
  int* cl_len;         // R^T pair lists: [slices] entries per slice of 64/Z cells
  long* cl_off;        // [slices] first entry of each slice
  int2* cl_ent;        // [entries][64/Z] (sample index, weight bits)
  float* symx;         // [n] 1 / (4 + 2 cos 2 pi k / n): the B-spline prefilter along the detector axis
};

namespace ht {
static cudaError_t build_cell_lists(ht_tomo_s* t);
}

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

static void tomo_free(ht_tomo_s* t) {
  cudaFree(t->phi);
  cudaFree(t->cs);
  cudaFree(t->th_sorted);
  cudaFree(t->th_index);
  cudaFree(t->fde);
  cudaFree(t->fab);
  cudaFree(t->gs);
  cudaFree(t->cl_len);
  cudaFree(t->cl_off);
  cudaFree(t->cl_ent);
  cudaFree(t->symx);
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
  std::vector<float> thm(ntheta);
  for (int i = 0; i < ntheta; ++i) {
    const double th = (double)theta_host[i];
    cs[i] = make_float2((float)std::cos(th), (float)std::sin(th));
    double r = std::fmod(th, M_PI);
    if (r < 0) r += M_PI;
    thm[i] = (float)r;
    if (thm[i] >= (float)M_PI) thm[i] = 0.f;
  }
  std::vector<int> idx(ntheta);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return thm[a] < thm[b]; });
  std::vector<float> ths(ntheta);
  for (int i = 0; i < ntheta; ++i) ths[i] = thm[idx[i]];
  t->tw_n = twiddle_table(n, t->device);
  t->tw_2n = twiddle_table(2 * n, t->device);
  const int Z = tomo_Z(n);
  const size_t nzp = (size_t)((nz + Z - 1) / Z) * Z;
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void** p, size_t b) {
    if (e == cudaSuccess) e = cudaMalloc(p, b);
  };
  alloc((void**)&t->phi, sizeof(float) * n * n);
  alloc((void**)&t->cs, sizeof(float2) * ntheta);
  alloc((void**)&t->th_sorted, sizeof(float) * ntheta);
  alloc((void**)&t->th_index, sizeof(int) * ntheta);
  alloc((void**)&t->fde, sizeof(float2) * nzp * 4 * n * n);
  alloc((void**)&t->fab, sizeof(float2) * nzp * 2 * n * n);
  alloc((void**)&t->gs, sizeof(float2) * nzp * ntheta * n);
  alloc((void**)&t->symx, sizeof(float) * n);
  std::vector<float> sx(n);
  for (int k = 0; k < n; ++k) sx[k] = (float)(1.0 / (4.0 + 2.0 * std::cos(2.0 * M_PI * k / n)));
  if (e == cudaSuccess) e = cudaMemcpy(t->phi, phi_host, sizeof(float) * n * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->cs, cs.data(), sizeof(float2) * ntheta, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->th_sorted, ths.data(), sizeof(float) * ntheta, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->th_index, idx.data(), sizeof(int) * ntheta, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t->symx, sx.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = build_cell_lists(t);
  if (e != cudaSuccess || !t->tw_n || !t->tw_2n) {
    if (e != cudaSuccess) set_error(std::string("ht_tomo_create: ") + cudaGetErrorString(e));
    tomo_free(t);
    delete t;
    return kCudaError;
  }
  *out = t;
  return kOk;
}

extern "C" int ht_tomo_destroy(ht_tomo_s* t) {
  if (!t) return ht::kOk;
  tomo_free(t);
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
  G.th_sorted = t->th_sorted;
  G.th_index = t->th_index;
  return G;
}

// The R^T pair lists (k_cell_count, k_slice_len, k_cell_fill) on a private
// stream; the per-cell counts use the Fourier-grid workspace as scratch.
static cudaError_t build_cell_lists(ht_tomo_s* t) {
  const GatherGeom G = geom(t);
  const int twon = 2 * t->n;
  const int cps = 64 / tomo_Z(t->n);
  const SliceShape sh = slice_shape(cps);
  const long ncells = (long)twon * twon, nsl = (long)((twon + sh.tw - 1) / sh.tw) * ((twon + sh.th - 1) / sh.th);
  int* cnt = reinterpret_cast<int*>(t->fde);
  cudaStream_t st = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e != cudaSuccess) return e;
  std::vector<int> len(nsl);
  std::vector<long> off(nsl);
  long tot = 0;
  e = cudaMalloc(&t->cl_len, sizeof(int) * nsl);
  if (e == cudaSuccess) e = cudaMalloc(&t->cl_off, sizeof(long) * nsl);
  if (e == cudaSuccess) {
    k_cell_count<<<(unsigned)((ncells + 255) / 256), 256, 0, st>>>(G, cnt);
    count_launch();
    k_slice_len<<<(unsigned)((nsl + 255) / 256), 256, 0, st>>>(cnt, twon, cps, t->cl_len, nsl);
    count_launch();
    e = cudaMemcpyAsync(len.data(), t->cl_len, sizeof(int) * nsl, cudaMemcpyDeviceToHost, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) {
    for (long i = 0; i < nsl; ++i) {
      off[i] = tot;
      tot += len[i];
    }
    e = cudaMemcpyAsync(t->cl_off, off.data(), sizeof(long) * nsl, cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaMalloc(&t->cl_ent, sizeof(int2) * cps * (size_t)std::max(tot, 1L));
  if (e == cudaSuccess) e = cudaMemsetAsync(t->cl_ent, 0, sizeof(int2) * cps * (size_t)std::max(tot, 1L), st);
  if (e == cudaSuccess) {
    k_cell_fill<<<(unsigned)((ncells + 255) / 256), 256, 0, st>>>(G, cps, t->cl_off, t->cl_ent);
    count_launch();
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return e;
}
}  // namespace ht

namespace ht {
static int tomo_R(ht_tomo_s* t, const void* obj, void* sino, int nz, int ldz, bool filt, void* stream) {
  HT_REQUIRE(t && obj && sino, "ht_tomo_R: null pointer");
  HT_REQUIRE(nz >= 0 && nz <= t->nz, "ht_tomo_R: nz exceeds the handle's slice capacity");
  HT_REQUIRE(ldz >= nz, "ht_tomo_R: ldz must be at least nz");
  if (nz == 0) return kOk;
  const GatherGeom G = geom(t);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float* symx = filt ? t->symx : nullptr;
  cudaError_t e = cudaErrorInvalidValue;
  switch (t->n) {
#define X(A, B)                                                                                             \
  case A:                                                                                                   \
    e = tomo_R_sized<B>(static_cast<const float2*>(obj), static_cast<float2*>(sino), t->phi, t->fab, t->fde, G, \
                        nz, ldz, t->tw_n, t->tw_2n, symx, st);                                              \
    break;
    HT_TOMO_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  return kOk;
}

static int tomo_RT(ht_tomo_s* t, const void* sino, void* obj, int nz, int ldz, bool filt, float scale,
                   void* stream) {
  HT_REQUIRE(t && obj && sino, "ht_tomo_RT: null pointer");
  HT_REQUIRE(nz >= 0 && nz <= t->nz, "ht_tomo_RT: nz exceeds the handle's slice capacity");
  HT_REQUIRE(ldz >= nz, "ht_tomo_RT: ldz must be at least nz");
  if (nz == 0) return kOk;
  const GatherGeom G = geom(t);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float* symx = filt ? t->symx : nullptr;
  cudaError_t e = cudaErrorInvalidValue;
  switch (t->n) {
#define X(A, B)                                                                                                 \
  case A:                                                                                                       \
    e = tomo_RT_sized<B>(static_cast<const float2*>(sino), static_cast<float2*>(obj), t->phi, t->fab, t->fde,    \
                         t->gs, G, CellLists{t->cl_len, t->cl_off, t->cl_ent}, nz, ldz, t->tw_n, t->tw_2n, symx, \
                         scale, st);                                                                                \
    break;
    HT_TOMO_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  return kOk;
}
}  // namespace ht

extern "C" int ht_tomo_R(ht_tomo_s* t, const void* obj, void* sino, int nz, void* stream) {
  return ht::tomo_R(t, obj, sino, nz, nz, false, stream);
}

extern "C" int ht_tomo_RT(ht_tomo_s* t, const void* sino, void* obj, int nz, void* stream) {
  return ht::tomo_RT(t, sino, obj, nz, nz, false, 1.0f, stream);
}

extern "C" int ht_tomo_R_coeffx(ht_tomo_s* t, const void* obj, void* sino, int nz, void* stream) {
  return ht::tomo_R(t, obj, sino, nz, nz, true, stream);
}

extern "C" int ht_tomo_RT_coeffx(ht_tomo_s* t, const void* sino, void* obj, int nz, float scale, void* stream) {
  return ht::tomo_RT(t, sino, obj, nz, nz, true, scale, stream);
}

extern "C" int ht_tomo_R_slab(ht_tomo_s* t, const void* obj, void* sino, int nz, int ldz, int coeffx, void* stream) {
  return ht::tomo_R(t, obj, sino, nz, ldz, coeffx != 0, stream);
}

extern "C" int ht_tomo_RT_slab(ht_tomo_s* t, const void* sino, void* obj, int nz, int ldz, int coeffx, float scale,
                               void* stream) {
  return ht::tomo_RT(t, sino, obj, nz, ldz, coeffx != 0, scale, stream);
}
