// Cubic B-spline shift family (reference: src/holotomocupy/shift.py:15-221,
// kernels src/holotomocupy/cuda_kernels.py:131-290, 377-843).
//
// coeff: the periodic B-spline prefilter ifft2(fft2(psi) / B3) of shift.py:74-82.
//   The symbol B3[ky,kx] = (4 + 2 cos 2pi ky/nzpsi)(4 + 2 cos 2pi kx/npsi) is a
//   product, so the filter runs as one row pass and one column pass, each an
//   FFT, a multiply by 1 / (N (4 + 2 cos 2pi k/N)) and an inverse FFT.
// S / dS / d2S: 4x4-tap stencils at the sample position
//   x = mag (tx - n/2) - r_x + (mag-1)/2 + npsi/2 (same for y with r_y, nz,
//   nzpsi), zero outside the coefficient grid (cuda_kernels.py:177-222).
// S^T and the object part of dS^T: the reference scatters with atomics; here
//   every coefficient gathers from the output pixels whose 4x4 footprint
//   contains it (found from the inverse of the monotone sample map and
//   re-checked with the forward formula), so results are deterministic.
// Position part of dS^T: per-angle sums Re<g, dS/dr_y c>, Re<g, dS/dr_x c>
//   reduced in double precision inside the kernel (no dt1/dt2 images).
// Element type T is float2 (complex64 objects) or float (float32 objects).
#include "lines.cuh"
#include "holotomo_b200_internal.h"

#include <cmath>
#include <vector>

namespace ht {

// ----------------------------------------------------------- the basis
// x6-scaled cubic B-spline and its derivatives (cuda_kernels.py:131-159)
__device__ __forceinline__ float bs0(float t) {
  if (-2.0f < t && t <= -1.0f) return (t + 2.0f) * (t + 2.0f) * (t + 2.0f);
  if (-1.0f < t && t <= 1.0f) return 4.0f - 6.0f * t * t + 3.0f * fabsf(t) * t * t;
  if (1.0f < t && t <= 2.0f) return (2.0f - t) * (2.0f - t) * (2.0f - t);
  return 0.0f;
}
__device__ __forceinline__ float bs1(float t) {
  if (-2.0f < t && t <= -1.0f) return 3.0f * (t + 2.0f) * (t + 2.0f);
  if (-1.0f < t && t <= 1.0f) return -12.0f * t + 9.0f * fabsf(t) * t;
  if (1.0f < t && t <= 2.0f) return -3.0f * (2.0f - t) * (2.0f - t);
  return 0.0f;
}
__device__ __forceinline__ float bs2(float t) {
  if (-2.0f < t && t <= -1.0f) return 6.0f * (t + 2.0f);
  if (-1.0f < t && t <= 1.0f) return -12.0f + 18.0f * fabsf(t);
  if (1.0f < t && t <= 2.0f) return 6.0f * (2.0f - t);
  return 0.0f;
}

// sample coordinate along one axis for output index t (cuda_kernels.py:179-184)
__device__ __forceinline__ float spline_x(float mag, int t, int nhalf, float shift, int npsihalf) {
  const float half = (mag - 1.0f) / 2.0f;
  return (mag * (float)(t - nhalf) - shift + half) + (float)npsihalf;
}

template <class T>
struct Ops;
template <>
struct Ops<float2> {
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ void fma(float2& a, float w, float2 v) {
    a.x += w * v.x;
    a.y += w * v.y;
  }
  static __device__ __forceinline__ float redot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
};
template <>
struct Ops<float> {
  static __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ void fma(float& a, float w, float v) { a += w * v; }
  static __device__ __forceinline__ float redot(float a, float b) { return a * b; }
};

struct ShiftDims {
  int n, npsi, nz, nzpsi;
};

// --------------------------------------------------- forward stencils
// MODE 0: S;  MODE 1: dS;  MODE 2: d2S
template <class T, int MODE>
__global__ void __launch_bounds__(256)
k_shift_stencil(T* __restrict__ out, const T* __restrict__ c, const T* __restrict__ c1, const T* __restrict__ c2,
                const float* __restrict__ r, const float* __restrict__ mag, const float* __restrict__ d1,
                const float* __restrict__ d2, ShiftDims D) {
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;
  const int b = blockIdx.z;
  if (tx >= D.n || ty >= D.nz) return;
  const float m0 = mag[b];
  const float x = spline_x(m0, tx, D.n / 2, r[2 * b + 1], D.npsi / 2);
  const float y = spline_x(m0, ty, D.nz / 2, r[2 * b + 0], D.nzpsi / 2);
  const int ix = (int)floorf(x), iy = (int)floorf(y);
  const float dx = x - (float)ix, dy = y - (float)iy;
  const long off = (long)b * D.npsi * D.nzpsi;
  float px[4], dpx[4], d2px[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float u = dx - (float)(j - 1);
    px[j] = bs0(u);
    if (MODE >= 1) dpx[j] = bs1(u);
    if (MODE == 2) d2px[j] = bs2(u);
  }
  float d1x = 0.f, d1y = 0.f, d2x = 0.f, d2y = 0.f, cross = 0.f;
  if (MODE >= 1) {
    d1x = d1[2 * b + 1];
    d1y = d1[2 * b + 0];
  }
  if (MODE == 2) {
    d2x = d2[2 * b + 1];
    d2y = d2[2 * b + 0];
    cross = d1x * d2y + d1y * d2x;
  }
  T acc = Ops<T>::zero();
#pragma unroll
  for (int jy = 0; jy < 4; ++jy) {
    const int yy = iy + jy - 1;
    if (yy < 0 || yy >= D.nzpsi) continue;
    const float u = dy - (float)(jy - 1);
    const float py = bs0(u);
    const float dpy = (MODE >= 1) ? bs1(u) : 0.f;
    const float d2py = (MODE == 2) ? bs2(u) : 0.f;
    const long rowoff = off + (long)yy * D.npsi;
#pragma unroll
    for (int jx = 0; jx < 4; ++jx) {
      const int xx = ix + jx - 1;
      if (xx < 0 || xx >= D.npsi) continue;
      const long idx = rowoff + xx;
      if (MODE == 0) {
        Ops<T>::fma(acc, px[jx] * py, __ldg(&c[idx]));
      } else if (MODE == 1) {
        // res = phi phi c1 - (phi'_x phi_y dr_x + phi_x phi'_y dr_y) c   (cuda_kernels.py:600-609)
        const float w = dpx[jx] * py * d1x + dpy * px[jx] * d1y;
        Ops<T>::fma(acc, -w, __ldg(&c[idx]));
        Ops<T>::fma(acc, px[jx] * py, __ldg(&c1[idx]));
      } else {
        // cuda_kernels.py:437-450 (c1 paired with d1, c2 with d2, as in the reference)
        const float w = d2px[jx] * py * d1x * d2x + dpx[jx] * dpy * cross + px[jx] * d2py * d1y * d2y;
        const float w1 = dpx[jx] * py * d1x + dpy * px[jx] * d1y;
        const float w2 = dpx[jx] * py * d2x + dpy * px[jx] * d2y;
        Ops<T>::fma(acc, w, __ldg(&c[idx]));
        Ops<T>::fma(acc, -w1, __ldg(&c1[idx]));
        Ops<T>::fma(acc, -w2, __ldg(&c2[idx]));
      }
    }
  }
  out[((long)b * D.nz + ty) * D.n + tx] = acc;
}

// ------------------------------------------------ adjoint (gather form)
// out[b, iy, ix] = sum over output pixels (ty, tx) whose footprint holds
// (iy, ix) of phi(dy - (iy - iy(ty))) phi(dx - (ix - ix(tx))) g[b, ty, tx].
// ADD: accumulate into out instead of overwriting.
__device__ __forceinline__ void cand_range(float m0, float C0, int i, int nhalf, int nmax, int& lo, int& hi) {
  // x(t) = m0 (t - nhalf) + C0 lies in [i-2, i+2).  A (near) zero
  // magnification maps every t to one point: all t are candidates.
  if (!(fabsf(m0) > 1e-3f)) {
    lo = 0;
    hi = nmax - 1;
    return;
  }
  float a = ((float)(i - 2) - C0) / m0 + (float)nhalf;
  float b = ((float)(i + 2) - C0) / m0 + (float)nhalf;
  const float l = fminf(fmaxf(fminf(a, b), -1e7f), 1e7f);
  const float h = fminf(fmaxf(fmaxf(a, b), -1e7f), 1e7f);
  lo = max(0, (int)floorf(l) - 1);
  hi = min(nmax - 1, (int)ceilf(h) + 1);
}

template <class T, bool ADD>
__global__ void __launch_bounds__(256)
k_shift_adj(T* __restrict__ out, const T* __restrict__ g, const float* __restrict__ r, const float* __restrict__ mag,
            ShiftDims D) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy = blockIdx.y * blockDim.y + threadIdx.y;
  const int b = blockIdx.z;
  if (ix >= D.npsi || iy >= D.nzpsi) return;
  const float m0 = mag[b];
  const float rx = r[2 * b + 1], ry = r[2 * b + 0];
  const float half = (m0 - 1.0f) / 2.0f;
  const float Cx = -rx + half + (float)(D.npsi / 2);
  const float Cy = -ry + half + (float)(D.nzpsi / 2);
  int tx0, tx1, ty0, ty1;
  cand_range(m0, Cx, ix, D.n / 2, D.n, tx0, tx1);
  cand_range(m0, Cy, iy, D.nz / 2, D.nz, ty0, ty1);
  const T* gb = g + (long)b * D.nz * D.n;
  T acc = Ops<T>::zero();
  for (int ty = ty0; ty <= ty1; ++ty) {
    const float y = spline_x(m0, ty, D.nz / 2, ry, D.nzpsi / 2);
    const int jy = iy - (int)floorf(y);
    if (jy < -1 || jy > 2) continue;
    const float wy = bs0(y - floorf(y) - (float)jy);
    T racc = Ops<T>::zero();
    for (int tx = tx0; tx <= tx1; ++tx) {
      const float x = spline_x(m0, tx, D.n / 2, rx, D.npsi / 2);
      const int jx = ix - (int)floorf(x);
      if (jx < -1 || jx > 2) continue;
      Ops<T>::fma(racc, bs0(x - floorf(x) - (float)jx), __ldg(&gb[(long)ty * D.n + tx]));
    }
    Ops<T>::fma(acc, wy, racc);
  }
  const long o = ((long)b * D.nzpsi + iy) * D.npsi + ix;
  if (ADD) {
    T prev = out[o];
    Ops<T>::fma(prev, 1.0f, acc);
    out[o] = prev;
  } else {
    out[o] = acc;
  }
}

// ------------------------------------- position part of the adjoint
// acc[b, 0] += sum Re<g, dt1>, acc[b, 1] += sum Re<g, dt2> with
// dt1 = sum -phi'_y phi_x c, dt2 = sum -phi'_x phi_y c (cuda_kernels.py:744-751)
template <class T>
__global__ void __launch_bounds__(256)
k_shift_dpos(double* __restrict__ acc, const T* __restrict__ c, const T* __restrict__ g, const float* __restrict__ r,
             const float* __restrict__ mag, ShiftDims D) {
  const int tx = blockIdx.x * blockDim.x + threadIdx.x;
  const int ty = blockIdx.y * blockDim.y + threadIdx.y;
  const int b = blockIdx.z;
  float s1 = 0.f, s2 = 0.f;
  if (tx < D.n && ty < D.nz) {
    const float m0 = mag[b];
    const float x = spline_x(m0, tx, D.n / 2, r[2 * b + 1], D.npsi / 2);
    const float y = spline_x(m0, ty, D.nz / 2, r[2 * b + 0], D.nzpsi / 2);
    const int ix = (int)floorf(x), iy = (int)floorf(y);
    const float dx = x - (float)ix, dy = y - (float)iy;
    const long off = (long)b * D.npsi * D.nzpsi;
    float px[4], dpx[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      px[j] = bs0(dx - (float)(j - 1));
      dpx[j] = bs1(dx - (float)(j - 1));
    }
    T a1 = Ops<T>::zero(), a2 = Ops<T>::zero();
#pragma unroll
    for (int jy = 0; jy < 4; ++jy) {
      const int yy = iy + jy - 1;
      if (yy < 0 || yy >= D.nzpsi) continue;
      const float py = bs0(dy - (float)(jy - 1));
      const float dpy = bs1(dy - (float)(jy - 1));
#pragma unroll
      for (int jx = 0; jx < 4; ++jx) {
        const int xx = ix + jx - 1;
        if (xx < 0 || xx >= D.npsi) continue;
        const T cv = __ldg(&c[off + (long)yy * D.npsi + xx]);
        Ops<T>::fma(a1, -dpy * px[jx], cv);
        Ops<T>::fma(a2, -dpx[jx] * py, cv);
      }
    }
    const T gv = g[((long)b * D.nz + ty) * D.n + tx];
    s1 = Ops<T>::redot(gv, a1);
    s2 = Ops<T>::redot(gv, a2);
  }
  // block reduction in double
  double v1 = s1, v2 = s2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v1 += __shfl_down_sync(0xffffffffu, v1, o);
    v2 += __shfl_down_sync(0xffffffffu, v2, o);
  }
  __shared__ double red[2][8];
  const int lin = threadIdx.y * blockDim.x + threadIdx.x;
  const int w = lin / 32, l = lin % 32;
  if (l == 0) {
    red[0][w] = v1;
    red[1][w] = v2;
  }
  __syncthreads();
  if (lin == 0) {
    double t1 = 0, t2 = 0;
    const int nw = (blockDim.x * blockDim.y + 31) / 32;
    for (int i = 0; i < nw; ++i) {
      t1 += red[0][i];
      t2 += red[1][i];
    }
    atomicAdd(&acc[2 * b + 0], t1);
    atomicAdd(&acc[2 * b + 1], t2);
  }
}

// ------------------------------------------- back-projection shift
// Sback (shift.py:138-148; cuda_kernels.py:294-370, dir = 1): the detector
// image g is spread onto the coefficient grid with the B-spline stretched by
// the image's magnification m.  Pixel (tx, ty) sits at
// x = (m (tx - n/2) - r_x + (m - 1)/2) + npsi/2 (y likewise), ix = floor(x),
// dx = x - ix, and reaches the cells ix + jx for jx in [ceil(dx - 2m),
// (int)(dx + 2m)) with weight phi((dx - jx) / m) (and the same in y; the upper
// bound drops the last tap of non-zero weight when dx + 2m is not an integer,
// as the reference has it).
//
// Here the transpose is a gather: one thread per coefficient cell finds the
// pixels whose tap windows contain it -- a window of about 4 + 2/m pixels
// around the cell's preimage, each tested with the exact membership rule
// above -- and sums their contributions in a fixed order (rows, then pixels
// within a row), so the result does not depend on scheduling and every cell
// is written once (no clearing pass, no atomics).
__device__ __forceinline__ float sback_phi(float t, float m) {
  t /= m;
  const float a = fabsf(t);
  if (t > -2.f && t <= -1.f) return (t + 2.f) * (t + 2.f) * (t + 2.f);
  if (t > -1.f && t <= 1.f) return 4.f - 6.f * t * t + 3.f * a * t * t;
  if (t > 1.f && t <= 2.f) return (2.f - t) * (2.f - t) * (2.f - t);
  return 0.f;
}

// Pixel p's position on the coefficient axis (the reference's float
// arithmetic) and whether its window reaches cell `cell`; *w is the tap weight.
__device__ __forceinline__ bool sback_tap(int p, int npix, int ncell, float shift, float m0, int cell, float* w) {
  const float half = (m0 - 1.0f) / 2.0f;
  const float x = (m0 * (float)(p - npix / 2) - shift + half) + (float)(ncell / 2);
  const int ix = (int)floorf(x);
  const float dx = x - (float)ix;
  const float span = 2.0f * m0;
  const int j = cell - ix;
  if (j < (int)ceilf(dx - span) || j >= (int)(dx + span)) return false;
  *w = sback_phi(dx - (float)j, m0);
  return true;
}

// The pixels whose windows can reach `cell`: sback_tap admits pixel p only
// when its position x(p) lies in (cell - 2m, cell + 2m], so p lies within
// (cell -+ 2m - c) / m + npix / 2; the range is widened by 0.01 cell units
// (far above the float rounding of x) and one pixel on each side, and
// membership is still decided by sback_tap.
__device__ __forceinline__ void sback_range(int cell, int npix, int ncell, float shift, float m0, int* p0, int* p1) {
  const float c = -shift + (m0 - 1.0f) / 2.0f + (float)(ncell / 2);
  const float lo = ((float)cell - 2.0f * m0 - 0.01f - c) / m0 + (float)(npix / 2);
  const float hi = ((float)cell + 2.0f * m0 + 0.01f - c) / m0 + (float)(npix / 2);
  *p0 = max(0, (int)floorf(fmaxf(lo, -1.0f)) - 1);
  *p1 = min(npix - 1, (int)ceilf(fminf(hi, (float)npix)) + 1);
}

// Candidate pixels a cell line's tap table holds; wider candidate ranges
// (very small magnifications) take the loop that tests them per pixel.
constexpr int kSbackX = 16;

// Tap table of one cell line: first candidate pixel, membership mask over
// the kSbackX candidates (bit 31: the candidate range is wider, the cell
// takes the per-pixel loop) and the weights.
__device__ __forceinline__ unsigned sback_taps(int cell, int npix, int ncell, float shift, float m0, int* p0,
                                               float (&w)[kSbackX]) {
  int p1;
  sback_range(cell, npix, ncell, shift, m0, p0, &p1);
  unsigned mask = 0u;
#pragma unroll
  for (int k = 0; k < kSbackX; ++k) w[k] = 0.f;
  if (p1 - *p0 >= kSbackX) return 1u << 31;
#pragma unroll
  for (int k = 0; k < kSbackX; ++k)
    if (*p0 + k <= p1 && sback_tap(*p0 + k, npix, ncell, shift, m0, cell, &w[k])) mask |= 1u << k;
  return mask;
}

// A CTA covers kSbackCX x kSbackCY cells of one image.  The x taps depend
// on the cell column only and the y taps on the cell row only, so the CTA
// forms them once -- the first warp the columns', the second the rows' --
// in shared memory; each cell then sums its rows of taps in the fixed order.
constexpr int kSbackCX = 32, kSbackCY = 8;

__global__ void __launch_bounds__(kSbackCX * kSbackCY)
k_sback(const float2* __restrict__ g, float2* __restrict__ f, const float* __restrict__ r,
        const float* __restrict__ mag, int nmag, ShiftDims S, long batch) {
  __shared__ float xw[kSbackX][kSbackCX], yw[kSbackX][kSbackCY];
  __shared__ int xp0[kSbackCX], yp0[kSbackCY];
  __shared__ unsigned xm[kSbackCX], ym[kSbackCY];
  const int xx = blockIdx.x * kSbackCX + threadIdx.x;
  const int yy = blockIdx.y * kSbackCY + threadIdx.y;
  const long b = blockIdx.z;
  const float m0 = mag[nmag == 1 ? 0 : b];
  const float ry = r[2 * b + 0], rx = r[2 * b + 1];
  const bool tapped = m0 > 0.f;   // m <= 0: the reference's tap ranges are empty
  if (threadIdx.y == 0) {
    int p0 = 0;
    float w[kSbackX];
    const unsigned mask = (tapped && xx < S.npsi) ? sback_taps(xx, S.n, S.npsi, rx, m0, &p0, w) : 0u;
    xp0[threadIdx.x] = p0;
    xm[threadIdx.x] = mask;
#pragma unroll
    for (int k = 0; k < kSbackX; ++k) xw[k][threadIdx.x] = (mask >> 31) ? 0.f : w[k];
  } else if (threadIdx.y == 1 && threadIdx.x < kSbackCY) {
    const int row = blockIdx.y * kSbackCY + threadIdx.x;
    int p0 = 0;
    float w[kSbackX];
    const unsigned mask = (tapped && row < S.nzpsi) ? sback_taps(row, S.nz, S.nzpsi, ry, m0, &p0, w) : 0u;
    yp0[threadIdx.x] = p0;
    ym[threadIdx.x] = mask;
#pragma unroll
    for (int k = 0; k < kSbackX; ++k) yw[k][threadIdx.x] = (mask >> 31) ? 0.f : w[k];
  }
  __syncthreads();
  if (xx >= S.npsi || yy >= S.nzpsi || b >= batch) return;
  float2 acc = make_float2(0.f, 0.f);
  const float2* gb = g + b * (long)S.nz * S.n;
  const unsigned mx = xm[threadIdx.x], my = ym[threadIdx.y];
  if (tapped && !((mx | my) >> 31)) {
    float wx[kSbackX];
#pragma unroll
    for (int k = 0; k < kSbackX; ++k) wx[k] = xw[k][threadIdx.x];
    const float2* g0 = gb + (long)yp0[threadIdx.y] * S.n + xp0[threadIdx.x];
    for (int ky = 0; ky < kSbackX; ++ky) {
      if (!((my >> ky) & 1u)) continue;
      const float wy = yw[ky][threadIdx.y];
      const float2* grow = g0 + (long)ky * S.n;
      float2 rsum = make_float2(0.f, 0.f);
#pragma unroll
      for (int kx = 0; kx < kSbackX; ++kx) {
        if (!((mx >> kx) & 1u)) continue;
        const float2 v = __ldg(&grow[kx]);
        rsum.x += wx[kx] * v.x;
        rsum.y += wx[kx] * v.y;
      }
      acc.x += wy * rsum.x;
      acc.y += wy * rsum.y;
    }
  } else if (tapped) {
    // a candidate range wider than the tables (very small magnifications)
    int tx0, tx1, ty0, ty1;
    sback_range(xx, S.n, S.npsi, rx, m0, &tx0, &tx1);
    sback_range(yy, S.nz, S.nzpsi, ry, m0, &ty0, &ty1);
    for (int ty = ty0; ty <= ty1; ++ty) {
      float wy;
      if (!sback_tap(ty, S.nz, S.nzpsi, ry, m0, yy, &wy)) continue;
      const float2* grow = gb + (long)ty * S.n;
      float2 rsum = make_float2(0.f, 0.f);
      for (int tx = tx0; tx <= tx1; ++tx) {
        float wx;
        if (!sback_tap(tx, S.n, S.npsi, rx, m0, xx, &wx)) continue;
        const float2 v = __ldg(&grow[tx]);
        rsum.x += wx * v.x;
        rsum.y += wx * v.y;
      }
      acc.x += wy * rsum.x;
      acc.y += wy * rsum.y;
    }
  }
  f[(b * S.nzpsi + yy) * (long)S.npsi + xx] = acc;
}

// -------------------------------------------------- prefilter passes
// data [nrows, N] in place: FFT, * sym[k], IFFT (sym carries 1/N)
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_symbol_rows(const float2* in, float2* out, long nrows, const float* __restrict__ sym,
              const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < nrows;
  SmRow sm{smem + line * SmRow::padded(N)};
  for (int k = t; k < N; k += T) sm.st(k, valid ? in[row * N + k] : make_float2(0.f, 0.f));
  __syncthreads();
  fft_line<N, false>(sm, t, tw4, line_sync<T>());
  for (int k = t; k < N; k += T) sm.st(k, cscale(sm.ld(k), __ldg(&sym[k])));
  __syncthreads();
  fft_line<N, true>(sm, t, tw4, line_sync<T>());
  if (!valid) return;
  for (int k = t; k < N; k += T) out[row * N + k] = sm.ld(k);
}

// data [nimg, N, ncols] in place along the column axis.  The forward FFT's
// first stage loads the block's C columns from global memory and the inverse
// FFT's last stage stores them back (a warp covers 32 / C rows of C adjacent
// columns per access); the tile passes shared memory only between stages.
template <int N>
__global__ void __launch_bounds__(ColCfg<N>::THREADS, ColCfg<N>::MIN_BLOCKS)
k_symbol_cols(const float2* in, float2* out, int ncols, const float* __restrict__ sym,
              const float2* __restrict__ tw4) {
  constexpr int C = ColCfg<N>::C;
  constexpr int T = ColCfg<N>::T;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const bool valid = blockIdx.x * C + c < ncols;
  const int col = min((int)blockIdx.x * C + c, ncols - 1);
  const long off = (long)blockIdx.y * N * ncols + col;
  SmCol<C> sm{tile + c};
  fft_line_from<N, false, typename ColCfg<N>::PL>(GColIn{in + off, ncols, valid}, sm, t, tw4);
  for (int k = t; k < N; k += T) sm.st(k, cscale(sm.ld(k), __ldg(&sym[k])));
  __syncthreads();
  fft_line_to<N, true, typename ColCfg<N>::PL>(sm, GColOut{out + off, ncols, valid}, t, tw4);
}

// The z pass at 512 rows: one 32-thread group per column, 16 samples a
// thread, radices 8-8-8.  Thread t holds butterflies t and t + 32 of the
// forward FFT's last stage (P = 64), i.e. samples b + 64 j, which are also
// the samples of the inverse FFT's first stage (P = 1) on the same
// butterflies: the symbol multiplies them in registers and the spectrum makes
// no round trip through shared memory between the two transforms.  The same
// butterflies as k_symbol_cols; the results agree to an ulp (the compiler
// may fuse a complex product's multiply-adds differently in the two).
constexpr int kSym512C = 8, kSym512Threads = 32 * kSym512C;

__global__ void __launch_bounds__(kSym512Threads)
k_symbol_cols512(const float2* in, float2* out, int ncols, const float* __restrict__ sym,
                 const float2* __restrict__ tw4) {
  constexpr int N = 512, E = 16, C = kSym512C;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const bool valid = blockIdx.x * C + c < ncols;
  const int col = min((int)blockIdx.x * C + c, ncols - 1);
  const long off = (long)blockIdx.y * N * ncols + col;
  SmCol<C> sm{tile + c};
  const CtaSync sync{};
  float2 v[E];
  // forward FFT: stage 1 (from global memory) and stage 2
  fft_stage<N, E, 8, 1, false, false, true>(v, SplitView<GColIn, SmCol<C>>{GColIn{in + off, ncols, valid}, sm}, t,
                                            tw4, sync);
  fft_stage<N, E, 8, 8, false, true, true>(v, sm, t, tw4, sync);
  // stage 3 (P = 64) kept in registers: v[8 s + j] = X[b_s + 64 j], b_s = t + 32 s; times the symbol
#pragma unroll
  for (int s2 = 0; s2 < 2; ++s2) {
    const int b = t + 32 * s2;
#pragma unroll
    for (int j = 0; j < 8; ++j) v[8 * s2 + j] = sm.ld(b + 64 * j);
    float2 w[8];
    twiddles<8, false>(tw4, b, N, w);
#pragma unroll
    for (int j = 1; j < 8; ++j) v[8 * s2 + j] = cmul(v[8 * s2 + j], w[j]);
    Dft<8, false>::run(&v[8 * s2]);
#pragma unroll
    for (int j = 0; j < 8; ++j) v[8 * s2 + j] = cscale(v[8 * s2 + j], __ldg(&sym[b + 64 * j]));
  }
  sync();  // every stage-3 load is done before the stores below
  // inverse FFT: stage 1 (P = 1) on the same butterflies, then stages 2 and 3 (to global memory)
#pragma unroll
  for (int s2 = 0; s2 < 2; ++s2) {
    const int b = t + 32 * s2;
    Dft<8, true>::run(&v[8 * s2]);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm.st(b * 8 + j, v[8 * s2 + j]);
  }
  sync();
  fft_stage<N, E, 8, 8, true, true, true>(v, sm, t, tw4, sync);
  fft_stage<N, E, 8, 64, true, false, false>(v, SplitView<SmCol<C>, GColOut>{sm, GColOut{out + off, ncols, valid}},
                                             t, tw4, sync);
}

template <int N>
static cudaError_t l_symbol_rows(const float2* in, float2* out, long nrows, const float* sym, const float2* tw,
                                 cudaStream_t st) {
  using CF = RowCfg<N>;
  cudaError_t e = allow_smem(k_symbol_rows<N>, CF::SMEM);
  if (e != cudaSuccess) return e;
  k_symbol_rows<N><<<(unsigned)((nrows + CF::LINES - 1) / CF::LINES), CF::THREADS, CF::SMEM, st>>>(in, out, nrows,
                                                                                                 sym, tw); ::ht::count_launch();
  return cudaGetLastError();
}

template <int N>
static cudaError_t l_symbol_cols(const float2* in, float2* out, long nimg, int ncols, const float* sym,
                                 const float2* tw, cudaStream_t st) {
  if constexpr (N == 512) {
    constexpr int smem = N * kSym512C * (int)sizeof(float2);
    k_symbol_cols512<<<dim3((ncols + kSym512C - 1) / kSym512C, (unsigned)nimg), kSym512Threads, smem, st>>>(
        in, out, ncols, sym, tw);
    ::ht::count_launch();
    return cudaGetLastError();
  }
  using CF = ColCfg<N>;
  cudaError_t e = allow_smem(k_symbol_cols<N>, CF::SMEM);
  if (e != cudaSuccess) return e;
  k_symbol_cols<N><<<dim3((ncols + CF::C - 1) / CF::C, (unsigned)nimg), CF::THREADS, CF::SMEM, st>>>(in, out, ncols,
                                                                                                   sym, tw);
  ::ht::count_launch();
  return cudaGetLastError();
}

cudaError_t symbol_rows(int N, const float2* in, float2* out, long nrows, const float* sym, const float2* tw,
                        cudaStream_t st) {
  switch (N) {
#define X(S) \
  case S:    \
    return l_symbol_rows<S>(in, out, nrows, sym, tw, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t symbol_cols(int N, const float2* in, float2* out, long nimg, int ncols, const float* sym,
                        const float2* tw, cudaStream_t st) {
  switch (N) {
#define X(S) \
  case S:    \
    return l_symbol_cols<S>(in, out, nimg, ncols, sym, tw, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace ht

// ================================================================= C ABI
struct ht_shift_s {
  int n, npsi, nz, nzpsi, is_complex, device;
  float* symx;  // [npsi]  1 / (npsi (4 + 2 cos 2 pi k / npsi))
  float* symy;  // [nzpsi]
  const float2* tw_x;
  const float2* tw_y;
};

extern "C" int ht_shift_create(int n, int npsi, int nz, int nzpsi, int is_complex, ht_shift_s** out) {
  using namespace ht;
  HT_REQUIRE(out != nullptr, "ht_shift_create: null pointer");
  HT_REQUIRE(n > 0 && npsi > 0 && nz > 0 && nzpsi > 0, "ht_shift_create: sizes must be positive");
  ht_shift_s* s = new ht_shift_s{n, npsi, nz, nzpsi, is_complex ? 1 : 0, 0, nullptr, nullptr, nullptr, nullptr};
  cudaGetDevice(&s->device);
  const bool fft_ok = fft_size_supported(npsi) && fft_size_supported(nzpsi);
  if (fft_ok) {
    s->tw_x = twiddle_table(npsi, s->device);
    s->tw_y = twiddle_table(nzpsi, s->device);
  }
  std::vector<float> hx(npsi), hy(nzpsi);
  for (int k = 0; k < npsi; ++k) hx[k] = (float)(1.0 / (npsi * (4.0 + 2.0 * std::cos(2.0 * M_PI * k / npsi))));
  for (int k = 0; k < nzpsi; ++k) hy[k] = (float)(1.0 / (nzpsi * (4.0 + 2.0 * std::cos(2.0 * M_PI * k / nzpsi))));
  cudaError_t e = cudaMalloc(&s->symx, sizeof(float) * npsi);
  if (e == cudaSuccess) e = cudaMalloc(&s->symy, sizeof(float) * nzpsi);
  if (e == cudaSuccess) e = cudaMemcpy(s->symx, hx.data(), sizeof(float) * npsi, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(s->symy, hy.data(), sizeof(float) * nzpsi, cudaMemcpyHostToDevice);
  if (e != cudaSuccess || (fft_ok && (!s->tw_x || !s->tw_y))) {
    if (e != cudaSuccess) set_error(std::string("ht_shift_create: ") + cudaGetErrorString(e));
    cudaFree(s->symx);
    cudaFree(s->symy);
    delete s;
    return kCudaError;
  }
  *out = s;
  return kOk;
}

extern "C" int ht_shift_destroy(ht_shift_s* s) {
  if (!s) return ht::kOk;
  cudaFree(s->symx);
  cudaFree(s->symy);
  delete s;
  return ht::kOk;
}

namespace {
ht::ShiftDims dims(const ht_shift_s* s) { return ht::ShiftDims{s->n, s->npsi, s->nz, s->nzpsi}; }
dim3 out_grid(const ht_shift_s* s, long batch) { return dim3((s->n + 31) / 32, (s->nz + 7) / 8, (unsigned)batch); }
dim3 coef_grid(const ht_shift_s* s, long batch) {
  return dim3((s->npsi + 31) / 32, (s->nzpsi + 7) / 8, (unsigned)batch);
}
const dim3 kBlock(32, 8);
}  // namespace

extern "C" int ht_shift_coeff(ht_shift_s* s, const void* psi, void* out, long batch, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && psi && out, "ht_shift_coeff: null pointer");
  HT_REQUIRE(s->is_complex, "ht_shift_coeff: works on complex64 data (pass real data as complex)");
  if (!fft_size_supported(s->npsi) || !fft_size_supported(s->nzpsi)) {
    set_error("ht_shift_coeff: npsi and nzpsi must be supported FFT lengths");
    return kUnsupported;
  }
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HT_CHECK_CUDA(symbol_rows(s->npsi, static_cast<const float2*>(psi), static_cast<float2*>(out),
                            batch * s->nzpsi, s->symx, s->tw_x, st));
  HT_CHECK_CUDA(symbol_cols(s->nzpsi, static_cast<float2*>(out), static_cast<float2*>(out), batch, s->npsi, s->symy,
                            s->tw_y, st));
  return kOk;
}

extern "C" int ht_shift_coeff_z(ht_shift_s* s, const void* in, void* out, long ncols, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && in && out, "ht_shift_coeff_z: null pointer");
  HT_REQUIRE(ncols >= 0, "ht_shift_coeff_z: ncols must be non-negative");
  if (!fft_size_supported(s->nzpsi)) {
    set_error("ht_shift_coeff_z: nzpsi must be a supported FFT length");
    return kUnsupported;
  }
  if (ncols == 0) return kOk;
  HT_REQUIRE(ncols <= 0x7fffffffL, "ht_shift_coeff_z: ncols too large");
  HT_CHECK_CUDA(symbol_cols(s->nzpsi, static_cast<const float2*>(in), static_cast<float2*>(out), 1, (int)ncols,
                            s->symy, s->tw_y, static_cast<cudaStream_t>(stream)));
  return kOk;
}

extern "C" int ht_shift_filter(ht_shift_s* s, const void* psi, void* out, long batch, const float* symx,
                               const float* symy, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && psi && out && symx && symy, "ht_shift_filter: null pointer");
  if (!fft_size_supported(s->npsi) || !fft_size_supported(s->nzpsi)) {
    set_error("ht_shift_filter: npsi and nzpsi must be supported FFT lengths");
    return kUnsupported;
  }
  HT_REQUIRE(batch >= 0, "ht_shift_filter: batch must be non-negative");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HT_CHECK_CUDA(symbol_rows(s->npsi, static_cast<const float2*>(psi), static_cast<float2*>(out), batch * s->nzpsi,
                            symx, s->tw_x, st));
  HT_CHECK_CUDA(symbol_cols(s->nzpsi, static_cast<float2*>(out), static_cast<float2*>(out), batch, s->npsi, symy,
                            s->tw_y, st));
  return kOk;
}

extern "C" int ht_shift_Sback(ht_shift_s* s, const void* g, const float* r, const float* mag, int nmag, void* out,
                              long batch, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && g && r && mag && out, "ht_shift_Sback: null pointer");
  HT_REQUIRE(nmag == 1 || nmag == batch, "ht_shift_Sback: nmag must be 1 or batch");
  HT_REQUIRE(batch >= 0 && batch <= 65535, "ht_shift_Sback: batch must be in [0, 65535]");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 sgrid((s->npsi + kSbackCX - 1) / kSbackCX, (s->nzpsi + kSbackCY - 1) / kSbackCY, (unsigned)batch);
  k_sback<<<sgrid, dim3(kSbackCX, kSbackCY), 0, st>>>(static_cast<const float2*>(g), static_cast<float2*>(out), r, mag,
                                                  nmag, dims(s), batch);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

template <int MODE>
static int shift_stencil(ht_shift_s* s, void* out, const void* c, const void* c1, const void* c2, const float* r,
                         const float* mag, const float* d1, const float* d2, long batch, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && out && c && r && mag, "shift: null pointer");
  HT_REQUIRE(MODE < 1 || (c1 && d1), "shift: null first-derivative operand");
  HT_REQUIRE(MODE < 2 || (c2 && d2), "shift: null second-derivative operand");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (s->is_complex) {
    k_shift_stencil<float2, MODE><<<out_grid(s, batch), kBlock, 0, st>>>(
        (float2*)out, (const float2*)c, (const float2*)c1, (const float2*)c2, r, mag, d1, d2, dims(s));
    ::ht::count_launch();
  }
  else {
    k_shift_stencil<float, MODE><<<out_grid(s, batch), kBlock, 0, st>>>(
        (float*)out, (const float*)c, (const float*)c1, (const float*)c2, r, mag, d1, d2, dims(s));
    ::ht::count_launch();
  }
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_shift_S(ht_shift_s* s, const void* c, const float* r, const float* mag, void* out, long batch,
                          void* stream) {
  return shift_stencil<0>(s, out, c, nullptr, nullptr, r, mag, nullptr, nullptr, batch, stream);
}

extern "C" int ht_shift_dS(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* c1,
                           const float* dr, void* out, long batch, void* stream) {
  return shift_stencil<1>(s, out, c, c1, nullptr, r, mag, dr, nullptr, batch, stream);
}

extern "C" int ht_shift_d2S(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* c1,
                            const float* dr1, const void* c2, const float* dr2, void* out, long batch,
                            void* stream) {
  return shift_stencil<2>(s, out, c, c1, c2, r, mag, dr1, dr2, batch, stream);
}

extern "C" int ht_shift_Sadj(ht_shift_s* s, const void* g, const float* r, const float* mag, void* out, long batch,
                             void* stream) {
  using namespace ht;
  HT_REQUIRE(s && g && r && mag && out, "ht_shift_Sadj: null pointer");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (s->is_complex) {
    k_shift_adj<float2, false><<<coef_grid(s, batch), kBlock, 0, st>>>((float2*)out, (const float2*)g, r, mag,
                                                                       dims(s));
    ::ht::count_launch();
  }
  else {
    k_shift_adj<float, false><<<coef_grid(s, batch), kBlock, 0, st>>>((float*)out, (const float*)g, r, mag, dims(s));
    ::ht::count_launch();
  }
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_shift_dSadj(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* g,
                              void* out1, double* out2, long batch, void* stream) {
  using namespace ht;
  HT_REQUIRE(s && c && r && mag && g && out1 && out2, "ht_shift_dSadj: null pointer");
  if (batch == 0) return kOk;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HT_CHECK_CUDA(cudaMemsetAsync(out2, 0, sizeof(double) * 2 * batch, st));
  if (s->is_complex) {
    k_shift_adj<float2, false><<<coef_grid(s, batch), kBlock, 0, st>>>((float2*)out1, (const float2*)g, r, mag,
                                                                       dims(s)); ::ht::count_launch();
    k_shift_dpos<float2><<<out_grid(s, batch), kBlock, 0, st>>>(out2, (const float2*)c, (const float2*)g, r, mag,
                                                                dims(s)); ::ht::count_launch();
  } else {
    k_shift_adj<float, false><<<coef_grid(s, batch), kBlock, 0, st>>>((float*)out1, (const float*)g, r, mag, dims(s)); ::ht::count_launch();
    k_shift_dpos<float><<<out_grid(s, batch), kBlock, 0, st>>>(out2, (const float*)c, (const float*)g, r, mag,
                                                               dims(s)); ::ht::count_launch();
  }
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

extern "C" int ht_filter_rows(int N, const void* in, void* out, long nrows, const float* sym, void* stream) {
  using namespace ht;
  HT_REQUIRE(in && out && sym, "ht_filter_rows: null pointer");
  if (!fft_size_supported(N)) {
    set_error("ht_filter_rows: unsupported row length");
    return kUnsupported;
  }
  if (nrows == 0) return kOk;
  int dev = 0;
  cudaGetDevice(&dev);
  const float2* tw = twiddle_table(N, dev);
  if (!tw) return kCudaError;
  HT_CHECK_CUDA(symbol_rows(N, static_cast<const float2*>(in), static_cast<float2*>(out), nrows, sym, tw,
                            static_cast<cudaStream_t>(stream)));
  return kOk;
}
