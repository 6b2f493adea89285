// Fused data-fidelity cascade of the Bilinear-Hessian solver
// (reference: src/holotomocupy/rec_mpi.py:250-353, 517-813).
//
// Forward model per angle theta and distance k (image img = theta*ndist + k):
//   x22 = S_{pos,mag}(c)            c = coeff(proj[theta]) (the B-spline
//                                   coefficients, cached by the caller)
//   x12 = exp(i x22),  x0 = D_k(prb[k] x12),  F = 1/N sum (|x0| - d)^2
// Gradient (rec_mpi.py:562-813): g0 = 2/N (x0 - d x0/|x0|), G = D_k^H g0,
//   P = G conj(x12) (cached), Y22 = -i conj(prb[k]) P (the gradient at x22),
//   grad prb[k] = sum_theta P, grad c[theta] = sum_k S_k^T Y22, and the
//   position gradient (-Ay, -Ax) with Ax = sum Re<Y22, (dS/dx) c>,
//   Ay = sum Re<Y22, (dS/dy) c>.
// Hessian form (rec_mpi.py:250-303).  With the cascade's second-order terms
// moved onto the gradient quantities, for directions y, z:
//   H(y, z) = 2/N sum [(1 - d/|x0|) Re(y0 conj z0) + d/|x0| Re(l0* y0) Re(l0* z0)]
//           + sum Re(conj(P) i (y_prb z22 + z_prb y22))       (second order of F1)
//           - sum Re(conj(P) prb y22 z22)                      (second order of F2)
//           + sum Re<Y22, d2S(c; c_y, r_y; c_z, r_z)>          (second order of F3)
// where y22 = dS(c, c_y, r_y), y0 = D_k(x12 (y_prb + i prb y22)), l0 = x0/|x0|.
// The F3 term is a bilinear form in the position directions with per-image
// coefficients Hxx, Hxy, Hyy (from c) and Ax, Ay of the direction's
// coefficients; the reference's d2s pairs c_y with r_y and c_z with r_z
// (exact when y = z), which ht_rec_hessian reports as H_ref(y, z) beside the
// symmetric H_sym(y, z) (c_y with r_z).  One Hessian pass over both
// directions costs two propagations per image; the reference's three
// cascades cost ten.
//
// Row kernels handle one detector row of one image per line, with the
// propagator's DCT passes fused in; the column passes are the propagator's.
#include "dct.cuh"
#include "row512.cuh"
#include "holotomo_b200_internal.h"

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

namespace ht {

// -------------------------------------------------------------- basics
// Cubic B-spline weights of the four taps j = 0..3 of a sample whose
// fractional offset is d in [0, 1): the reference's piecewise kernels
// (cuda_kernels.py:8-60) evaluated at t = d + 1, d, d - 1, d - 2, with the
// branch of each tap fixed (e = 1 - d).
__device__ __forceinline__ void bw0(float d, float (&w)[4]) {
  const float e = 1.0f - d, d2 = d * d, e2 = e * e;
  w[0] = e2 * e;
  w[1] = 4.0f - 6.0f * d2 + 3.0f * d2 * d;
  w[2] = 4.0f - 6.0f * e2 + 3.0f * e2 * e;
  w[3] = d2 * d;
}
__device__ __forceinline__ void bw1(float d, float (&w)[4]) {
  const float e = 1.0f - d;
  w[0] = -3.0f * e * e;
  w[1] = -12.0f * d + 9.0f * d * d;
  w[2] = 12.0f * e - 9.0f * e * e;
  w[3] = 3.0f * d * d;
}
__device__ __forceinline__ void bw2(float d, float (&w)[4]) {
  const float e = 1.0f - d;
  w[0] = 6.0f * e;
  w[1] = -12.0f + 18.0f * d;
  w[2] = -12.0f + 18.0f * e;
  w[3] = 6.0f * d;
}

// Object-side element: complex (complex64 objects) or real (float32 objects)
template <class T>
struct El;
template <>
struct El<float2> {
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  // one packed two-lane FMA (the stencil taps' real weight on a complex sample)
  static __device__ __forceinline__ void fma(float2& a, float w, float2 v) {
#if defined(__CUDA_ARCH__)
    a = p2_fma(make_float2(w, w), v, a);
#endif
  }

  static __device__ __forceinline__ float2 cplx(float2 v) { return v; }
  // projection of a complex gradient onto the element space
  static __device__ __forceinline__ float2 proj(float2 g) { return g; }
  static __device__ __forceinline__ float2 from_sm(float2 g) { return g; }
  static __device__ __forceinline__ float redot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
};
template <>
struct El<float> {
  static __device__ __forceinline__ float zero() { return 0.f; }
  static __device__ __forceinline__ void fma(float& a, float w, float v) { a += w * v; }
  static __device__ __forceinline__ float2 cplx(float v) { return make_float2(v, 0.f); }
  static __device__ __forceinline__ float proj(float2 g) { return g.x; }
  static __device__ __forceinline__ float from_sm(float2 g) { return g.x; }
  static __device__ __forceinline__ float redot(float a, float b) { return a * b; }
};

// exp(i z) for complex z = a + ib: exp(-b) (cos a + i sin a)
__device__ __forceinline__ float2 cexp_i(float2 z) {
  float s, c;
  sincosf(z.x, &s, &c);
  const float e = expf(-z.y);
  return make_float2(e * c, e * s);
}

struct CascDims {
  int n, nz, nobj, nzobj, ndist;
  long nimg;         // ntheta * ndist
  int shared_c = 0;  // 1: one coefficient array [nzobj, nobj] for every angle
};

// Offset of angle th's coefficient array.
__device__ __forceinline__ long coef_off(const CascDims& D, long th) {
  return D.shared_c ? 0 : th * (long)D.nzobj * D.nobj;
}

// Object coordinate of detector column tx / row ty (cuda_kernels.py:177-190):
// mag * (t - n/2) - shift + (mag - 1)/2 + nobj/2.  Forward and adjoint use
// these same expressions, so the stencil footprints agree exactly.
__device__ __forceinline__ float sample_x(const CascDims& D, float mag, float rx, int tx) {
  return (mag * (float)(tx - D.n / 2) - rx + (mag - 1.0f) / 2.0f) + (float)(D.nobj / 2);
}
__device__ __forceinline__ float sample_y(const CascDims& D, float mag, float ry, int ty) {
  return (mag * (float)(ty - D.nz / 2) - ry + (mag - 1.0f) / 2.0f) + (float)(D.nzobj / 2);
}

// Vertical stencil of one detector row: the four object rows it reads
// (clamped into range; taps outside the object get weight 0) and their
// weights.  The whole detector row shares it.
template <int ORDER>
struct RowGeo {
  int yy[4];
  float py[4], dpy[4], d2py[4];
  __device__ __forceinline__ RowGeo(const CascDims& D, float mag, float ry, int ty) {
    const float y = sample_y(D, mag, ry, ty);
    const int iy = (int)floorf(y);
    const float dy = y - (float)iy;
    bw0(dy, py);
    if (ORDER >= 1) bw1(dy, dpy);
    if (ORDER >= 2) bw2(dy, d2py);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = iy + j - 1;
      const bool in = r >= 0 && r < D.nzobj;
      yy[j] = in ? r : 0;
      if (!in) {
        py[j] = 0.f;
        if (ORDER >= 1) dpy[j] = 0.f;
        if (ORDER >= 2) d2py[j] = 0.f;
      }
    }
  }
};

// Horizontal stencil of one detector pixel (same conventions).
template <int ORDER>
struct ColGeo {
  int xx[4];
  float px[4], dpx[4], d2px[4];
  __device__ __forceinline__ ColGeo(const CascDims& D, float mag, float rx, int tx) {
    const float x = sample_x(D, mag, rx, tx);
    const int ix = (int)floorf(x);
    const float dx = x - (float)ix;
    bw0(dx, px);
    if (ORDER >= 1) bw1(dx, dpx);
    if (ORDER >= 2) bw2(dx, d2px);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = ix + j - 1;
      const bool in = c >= 0 && c < D.nobj;
      xx[j] = in ? c : 0;
      if (!in) {
        px[j] = 0.f;
        if (ORDER >= 1) dpx[j] = 0.f;
        if (ORDER >= 2) d2px[j] = 0.f;
      }
    }
  }
};

template <class T>
__device__ __forceinline__ T dot4(const float (&w)[4], const T (&v)[4]) {
  T a = El<T>::zero();
#pragma unroll
  for (int j = 0; j < 4; ++j) El<T>::fma(a, w[j], v[j]);
  return a;
}

__device__ __forceinline__ float2 ld_pos(const float* pos, long img) {
  return make_float2(pos[2 * img + 0], pos[2 * img + 1]);
}

// Doubles of shared scratch line_sums<T, K> needs for a block of THREADS,
// rounded up to an even count so that what follows it stays 16-byte aligned.
template <int T>
__host__ __device__ constexpr int red_doubles(int K, int threads) {
  return ((T % 32 == 0 ? K * (threads / 32) : K * threads) + 1) / 2 * 2;
}

// Launch shape of a stencil row kernel: NFFT row lines of the DCT plus NSET
// vertically reduced object rows (nobj <= N values each) per detector row,
// with as many detector rows per CTA as keep the shared memory near 100 KB.
// A detector row has TR = NFFT * T threads: the stencil work is spread over
// all of them and each group of T transforms one of the row's NFFT lines, so
// the threads per SM grow with the row's shared memory.
template <int N, int NSET, int NFFT>
struct StCfg {
  using PL = StPlan<N>;
  static constexpr int T = PL::T;
  static constexpr int TR = NFFT * T;
  static constexpr int PER_LINE = NFFT * SmRow::padded(N) * 8 + NSET * N * 8;
  static constexpr int fit(int l) { return (l > 1 && l * PER_LINE > 100 * 1024) ? fit(l / 2) : l; }
  static constexpr int ROW_LINES = (T >= 256) ? 1 : (256 / T);  // lines a CTA of plain row lines holds
  static constexpr int LINES = fit(ROW_LINES / NFFT > 0 ? ROW_LINES / NFFT : 1);
  static constexpr int THREADS = LINES * TR;
  // each FFT group of T threads is a line with its own named barrier (1..15)
  static_assert(T % 32 != 0 || LINES * NFFT <= 15, "at most 15 line barriers per block");
  // dynamic shared memory: FFT lines, then reduction scratch, then the rows
  static constexpr int FFT_BYTES = LINES * NFFT * SmRow::padded(N) * 8;
  static int bytes(int K, int nobj, int elem) {
    return FFT_BYTES + red_doubles<TR>(K, THREADS) * 8 + LINES * NSET * nobj * elem;
  }
};

// Vertical pass of a detector row: V[s][ix] = sum_jy w_s[jy] c[yy[jy], ix]
// for the weight sets w_s of the row (every object column ix, by the T threads
// of the line).  The horizontal taps then read V from shared memory.
template <class T, int NS>
__device__ __forceinline__ void vrows(T* __restrict__ V, int nobj, const T* __restrict__ cb, const int (&yy)[4],
                                      const float* const (&w)[NS], int t, int TT) {
  const T* r0 = cb + (long)yy[0] * nobj;
  const T* r1 = cb + (long)yy[1] * nobj;
  const T* r2 = cb + (long)yy[2] * nobj;
  const T* r3 = cb + (long)yy[3] * nobj;
  for (int ix = t; ix < nobj; ix += TT) {
    const T v0 = __ldg(&r0[ix]), v1 = __ldg(&r1[ix]), v2 = __ldg(&r2[ix]), v3 = __ldg(&r3[ix]);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      T a = El<T>::zero();
      El<T>::fma(a, w[k][0], v0);
      El<T>::fma(a, w[k][1], v1);
      El<T>::fma(a, w[k][2], v2);
      El<T>::fma(a, w[k][3], v3);
      V[k * nobj + ix] = a;
    }
  }
}

// the four samples of a vertically reduced row under a pixel's stencil
template <class T>
__device__ __forceinline__ void vrow4(const T* __restrict__ V, const int (&xx)[4], T (&v)[4]) {
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = V[xx[j]];
}

// Two adjacent elements of T moved as one vector (16 bytes for complex, 8 for
// real): the interleaved vertical rows store the sets of one object column
// side by side, so a tap's sets load in NS / 2 accesses.
template <class T>
struct Pair;
template <>
struct Pair<float2> {
  static __device__ __forceinline__ void st(float2* p, float2 a, float2 b) {
    *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
  }
  static __device__ __forceinline__ void ld(const float2* p, float2& a, float2& b) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    a = make_float2(q.x, q.y);
    b = make_float2(q.z, q.w);
  }
};
template <>
struct Pair<float> {
  static __device__ __forceinline__ void st(float* p, float a, float b) {
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
  }
  static __device__ __forceinline__ void ld(const float* p, float& a, float& b) {
    const float2 q = *reinterpret_cast<const float2*>(p);
    a = q.x;
    b = q.y;
  }
};

// vrows for two weight sets into the interleaved layout V[ix * NST + base + {0, 1}]
// (the same sums, in the same order, as vrows)
template <class T, int NST>
__device__ __forceinline__ void vrows_pair(T* __restrict__ V, int base, int nobj, const T* __restrict__ cb,
                                           const int (&yy)[4], const float* __restrict__ w0,
                                           const float* __restrict__ w1, int t, int TT) {
  const T* r0 = cb + (long)yy[0] * nobj;
  const T* r1 = cb + (long)yy[1] * nobj;
  const T* r2 = cb + (long)yy[2] * nobj;
  const T* r3 = cb + (long)yy[3] * nobj;
  for (int ix = t; ix < nobj; ix += TT) {
    const T v0 = __ldg(&r0[ix]), v1 = __ldg(&r1[ix]), v2 = __ldg(&r2[ix]), v3 = __ldg(&r3[ix]);
    T a = El<T>::zero(), b = El<T>::zero();
    El<T>::fma(a, w0[0], v0);
    El<T>::fma(a, w0[1], v1);
    El<T>::fma(a, w0[2], v2);
    El<T>::fma(a, w0[3], v3);
    El<T>::fma(b, w1[0], v0);
    El<T>::fma(b, w1[1], v1);
    El<T>::fma(b, w1[2], v2);
    El<T>::fma(b, w1[3], v3);
    Pair<T>::st(V + (long)ix * NST + base, a, b);
  }
}

// Per-image accumulator slots
enum Acc : int { kAx = 0, kAy, kHxx, kHxy, kHyy, kAyx, kAyy, kAzx, kAzy, kNAcc };
// Global accumulator slots
enum Glob : int { kF = 0, kQ0, kQ1, kQ2, kL10, kL11, kL12, kL20, kL21, kL22, kNGlob };
// Per-row sum slots the row kernels write (see k_rows_img)
constexpr int kHessRowK = 10;  // the Hessian row pass's slots
constexpr int kRowKMax = 10;
constexpr int kRedThreads = 256;

// ================================================= forward row pass
// u = prb[k] exp(i S(c)) -> row DCT-II -> tmp
template <int N, class T>
__global__ void __launch_bounds__(StCfg<N, 1, 1>::THREADS, 4)
k_casc_fwd(const T* __restrict__ c, const float* __restrict__ pos, const float* __restrict__ mag,
           const float2* __restrict__ prb, float2* __restrict__ tmp, CascDims D, const float2* __restrict__ tw4) {
  using CF = StCfg<N, 1, 1>;
  constexpr int TT = CF::T;
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / TT, t = threadIdx.x % TT;
  const long row = (long)blockIdx.x * CF::LINES + line;  // img * nz + ty
  const bool valid = row < D.nimg * D.nz;
  const long img = valid ? row / D.nz : 0;
  const int ty = valid ? (int)(row % D.nz) : 0;
  const int k = (int)(img % D.ndist);
  const long th = img / D.ndist;
  SmRow sm{smem + line * SmRow::padded(N)};
  T* V = reinterpret_cast<T*>(reinterpret_cast<char*>(smem) + CF::FFT_BYTES) + (long)line * D.nobj;
  const float m0 = valid ? mag[img] : 1.f;
  const float2 r = valid ? ld_pos(pos, img) : make_float2(0.f, 0.f);
  const RowGeo<0> rg(D, m0, r.x, ty);
  if (valid) {
    const float* const w[1] = {rg.py};
    vrows<T, 1>(V, D.nobj, c + coef_off(D, th), rg.yy, w, t, TT);
  }
  __syncthreads();
  for (int tx = t; tx < N; tx += TT) {
    float2 u = make_float2(0.f, 0.f);
    if (valid) {
      const ColGeo<0> cg(D, m0, r.y, tx);
      T v[4];
      vrow4(V, cg.xx, v);
      const T x22 = dot4(cg.px, v);
      u = cmul(prb[((long)k * D.nz + ty) * N + tx], cexp_i(El<T>::cplx(x22)));
    }
    dct2_put<N>(sm, tx, u);
  }
  __syncthreads();
  dct2_finish<N, TT, typename CF::PL>(sm, t, tw4, tmp + row * N, valid);
}

// ======================================== residual row pass
// tmp holds the column-processed spectrum of u.  MODE 0: x0 -> cache,
// F, g0 -> DCT-II -> tmp.  MODE 1: F only.  MODE 2: out = |x0| (float).
template <int N, int MODE>
__global__ void __launch_bounds__(RowCfg<N>::THREADS, 4)
k_casc_resid(float2* __restrict__ tmp, float2* __restrict__ x0c, const float* __restrict__ data,
             float* __restrict__ amp, double* __restrict__ glob, double* __restrict__ rows, float scale,
             CascDims D, const float2* __restrict__ tw4) {
  constexpr int TT = RowCfg<N>::T;
  constexpr int E = Plan<N>::E;
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(smem + RowCfg<N>::LINES * SmRow::padded(N));
  const int line = threadIdx.x / TT, t = threadIdx.x % TT;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < D.nimg * D.nz;
  SmRow sm{smem + line * SmRow::padded(N)};
  // the data row is loaded before the transform, so its latency overlaps it
  float dv[E];
#pragma unroll
  for (int i = 0; i < E; ++i) dv[i] = (MODE != 2 && valid) ? data[row * N + t + i * TT] : 0.f;
  dct3_start<N, TT>(sm, t, tw4, tmp + row * N, valid);
  float2 g0[E];
  double acc[1] = {0.0};
  float facc = 0.f;
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int tx = t + i * TT;
    g0[i] = make_float2(0.f, 0.f);
    if (valid) {
      const float2 x0 = sm.ld(dct_perm(tx, N));
      const float a = sqrtf(x0.x * x0.x + x0.y * x0.y);
      if (MODE == 2) {
        amp[row * N + tx] = a;
      } else {
        const float d = dv[i];
        const float e = a - d;
        facc += e * e;
        if (MODE == 0) {
          x0c[row * N + tx] = x0;
          // rec_mpi.py:557-559: scale * (x - y * (x / |x|))
          const float2 l = make_float2(x0.x / a, x0.y / a);
          g0[i] = make_float2(scale * (x0.x - d * l.x), scale * (x0.y - d * l.y));
        }
      }
    }
  }
  if (MODE != 2) {
    acc[0] = facc;
    line_sums<TT, 1>(acc, red, line, t);
    if (t == 0 && valid) {
      if (rows)
        rows[row] = acc[0];  // summed by k_rows_img / k_imgs_glob
      else
        atomicAdd(&glob[kF], acc[0]);
    }
  }
  if (MODE != 0) return;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < E; ++i) dct2_put<N>(sm, t + i * TT, g0[i]);
  __syncthreads();
  dct2_finish<N, TT>(sm, t, tw4, tmp + row * N, valid);
}

// ------------------------------------------- 512-sample rows, a warp a row
// k_casc_resid and k_casc_hess_q at N = 512 on the warp-per-line transforms
// of row512.cuh: the DCT-III's pixels stay in registers for the residual and
// go on to the DCT-II from there, and the row sums are warp reductions.
constexpr int kR512Lines = 4;  // rows (warps) per block

template <int MODE>
__global__ void __launch_bounds__(32 * kR512Lines)
k_casc_resid512(float2* __restrict__ tmp, float2* __restrict__ x0c, const float* __restrict__ data,
                float* __restrict__ amp, double* __restrict__ glob, double* __restrict__ rows, float scale,
                CascDims D, const float2* __restrict__ tw4) {
  constexpr int N = kR512;
  __shared__ float2 smem[kR512Lines * SmRow::padded(N)];
  const int line = threadIdx.x / 32, t = threadIdx.x % 32;
  const long row = (long)blockIdx.x * kR512Lines + line;
  const bool valid = row < D.nimg * D.nz;
  SmRow sm{smem + line * SmRow::padded(N)};
  // the data row is loaded first, so its latency overlaps the transform
  float dv[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) dv[i] = (MODE != 2 && valid) ? data[row * N + dct_sample_at(r512_pos(t, i), N)] : 0.f;
  float2 v[16];
  r512_dct3_head(v, tmp + row * N, valid, sm, t, tw4);
  r512_finish_to_regs(v, sm, t, tw4);
  float facc = 0.f;
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int tx = dct_sample_at(r512_pos(t, i), N);
    const float2 x0 = v[i];
    v[i] = make_float2(0.f, 0.f);
    if (!valid) continue;
    const float a = sqrtf(x0.x * x0.x + x0.y * x0.y);
    if (MODE == 2) {
      amp[row * N + tx] = a;
    } else {
      const float d = dv[i];
      const float e = a - d;
      facc += e * e;
      if (MODE == 0) {
        x0c[row * N + tx] = x0;
        // rec_mpi.py:557-559: scale * (x - y * (x / |x|))
        const float2 l = make_float2(x0.x / a, x0.y / a);
        v[i] = make_float2(scale * (x0.x - d * l.x), scale * (x0.y - d * l.y));
      }
    }
  }
  if (MODE != 2) {
    const double acc = warp_sum((double)facc);
    if (t == 0 && valid) {
      if (rows)
        rows[row] = acc;
      else
        atomicAdd(&glob[kF], acc);
    }
  }
  if (MODE != 0) return;
  r512_dct2_tail(v, sm, t, tw4, tmp + row * N, valid);
}

template <int NDIR>
__global__ void __launch_bounds__(32 * kR512Lines, 6)
k_casc_hess_q512(const float2* __restrict__ tmp, const float2* __restrict__ x0c, const float* __restrict__ data,
                 double* __restrict__ rows, CascDims D, const float2* __restrict__ tw4) {
  constexpr int N = kR512;
  __shared__ float2 smem[NDIR * kR512Lines * SmRow::padded(N)];
  const int line = threadIdx.x / 32, t = threadIdx.x % 32;
  const long row = (long)blockIdx.x * kR512Lines + line;
  const long nrow = D.nimg * D.nz;
  const bool valid = row < nrow;
  SmRow sm0{smem + line * SmRow::padded(N)};
  SmRow sm1{smem + (NDIR - 1) * kR512Lines * SmRow::padded(N) + line * SmRow::padded(N)};
  // the rows read after the first transform (the second direction's
  // spectrum, x0 and the data) are brought into L2 now
  if (t == 0 && valid) {
    if (NDIR == 2) l2_prefetch(tmp + (nrow + row) * N, N * sizeof(float2));
    l2_prefetch(x0c + row * N, N * sizeof(float2));
    l2_prefetch(data + row * N, N * sizeof(float));
  }
  float2 v[16];
  r512_dct3_head(v, tmp + row * N, valid, sm0, t, tw4);
  r512_finish_to_regs(v, sm0, t, tw4);
  if (NDIR == 2) {
    // direction 0's pixels go back to sm0 (each thread its own positions)
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 16; ++i) sm0.st(r512_pos(t, i), v[i]);
    r512_dct3_head(v, tmp + (nrow + row) * N, valid, sm1, t, tw4);
    r512_finish_to_regs(v, sm1, t, tw4);
  }
  float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    if (!valid) break;
    const int tx = dct_sample_at(r512_pos(t, i), N);
    const float2 x0 = x0c[row * N + tx];
    const float d = data[row * N + tx];
    const float a = sqrtf(x0.x * x0.x + x0.y * x0.y);
    const float2 l0 = make_float2(x0.x / a, x0.y / a);
    const float d0 = d / a;
    const float2 y0 = (NDIR == 2) ? sm0.ld(r512_pos(t, i)) : v[i];
    const float ly = l0.x * y0.x + l0.y * y0.y;  // Re(conj(l0) y0)
    s[0] += (1.f - d0) * (y0.x * y0.x + y0.y * y0.y) + d0 * ly * ly;
    if (NDIR == 2) {
      const float2 y1 = v[i];
      const float lz = l0.x * y1.x + l0.y * y1.y;
      s[1] += (1.f - d0) * (y0.x * y1.x + y0.y * y1.y) + d0 * ly * lz;
      s[2] += (1.f - d0) * (y1.x * y1.x + y1.y * y1.y) + d0 * lz * lz;
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double x = warp_sum((double)s[i]);
    if (t == 0 && valid) rows[row * 3 + i] = x;  // Q0, Q1, Q2: k_rows_img / k_imgs_glob
  }
}

// Detector columns [lo, hi] whose stencil can reach object index i (a
// superset; callers test the exact footprint).  C0 is the coordinate offset
// and nhalf the detector half size of the axis.
__device__ __forceinline__ void cand_range(float m0, float C0, int i, int nhalf, int nmax, int& lo, int& hi) {
  if (!(fabsf(m0) > 1e-3f)) {
    lo = 0;
    hi = nmax - 1;
    return;
  }
  const float a = ((float)(i - 2) - C0) / m0 + (float)nhalf;
  const float b = ((float)(i + 2) - C0) / m0 + (float)nhalf;
  const float l = fminf(fmaxf(fminf(a, b), -1e7f), 1e7f);
  const float h = fminf(fmaxf(fmaxf(a, b), -1e7f), 1e7f);
  lo = max(0, (int)floorf(l) - 1);
  hi = min(nmax - 1, (int)ceilf(h) + 1);
}

// cand_range with the reciprocal rm0 = 1 / m0 computed once (0 when
// |m0| <= 1e-3: every index is a candidate).  The quotient moves by an ulp at
// most, well inside the one-index margin on either side.
__device__ __forceinline__ float cand_rm0(float m0) { return (fabsf(m0) > 1e-3f) ? 1.0f / m0 : 0.f; }
__device__ __forceinline__ void cand_range_r(float rm0, float C0, int i, int nhalf, int nmax, int& lo, int& hi) {
  if (rm0 == 0.f) {
    lo = 0;
    hi = nmax - 1;
    return;
  }
  const float a = ((float)(i - 2) - C0) * rm0 + (float)nhalf;
  const float b = ((float)(i + 2) - C0) * rm0 + (float)nhalf;
  const float l = fminf(fmaxf(fminf(a, b), -1e7f), 1e7f);
  const float h = fminf(fmaxf(fmaxf(a, b), -1e7f), 1e7f);
  lo = max(0, (int)floorf(l) - 1);
  hi = min(nmax - 1, (int)ceilf(h) + 1);
}

// The adjoint's horizontal gather reads, per detector pixel, the first object
// column of its stencil (int) and its four tap weights (float): 20 bytes, kept
// where the vertically reduced rows were once those are consumed.  Elements of
// T per detector row of that shared area:
// The vertical rows themselves: set 0 as nobj elements, then sets 1 and 2
// as nobj pairs from an even offset (so that a pair loads as one vector).
constexpr int kAdjTabBytes = 20;
__host__ __device__ constexpr int adj_pair_off(int nobj) { return (nobj + 1) / 2 * 2; }
__host__ __device__ constexpr int adj_line_elems(int nobj, int n, int elem) {
  return ((adj_pair_off(nobj) + 2 * nobj) * elem >= kAdjTabBytes * n)
             ? adj_pair_off(nobj) + 2 * nobj
             : ((kAdjTabBytes * n + elem - 1) / elem + 1) / 2 * 2;
}

// vrows for the adjoint's three weight sets: set 0 to V0[ix], sets 1 and 2 to
// the pair V12[2 ix], V12[2 ix + 1] (the sums and their order as in vrows)
template <class T>
__device__ __forceinline__ void vrows_adj(T* __restrict__ V0, T* __restrict__ V12, int nobj,
                                          const T* __restrict__ cb, const int (&yy)[4],
                                          const float* const (&w)[3], int t, int TT) {
  const T* r0 = cb + (long)yy[0] * nobj;
  const T* r1 = cb + (long)yy[1] * nobj;
  const T* r2 = cb + (long)yy[2] * nobj;
  const T* r3 = cb + (long)yy[3] * nobj;
  for (int ix = t; ix < nobj; ix += TT) {
    const T v0 = __ldg(&r0[ix]), v1 = __ldg(&r1[ix]), v2 = __ldg(&r2[ix]), v3 = __ldg(&r3[ix]);
    T a[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      a[k] = El<T>::zero();
      El<T>::fma(a[k], w[k][0], v0);
      El<T>::fma(a[k], w[k][1], v1);
      El<T>::fma(a[k], w[k][2], v2);
      El<T>::fma(a[k], w[k][3], v3);
    }
    V0[ix] = a[0];
    Pair<T>::st(V12 + 2 * ix, a[1], a[2]);
  }
}

// ============================================== adjoint row pass
// tmp holds the column-processed spectrum of g0.  G = DCT-III; recompute
// x12; P = G conj(x12) -> cache; Y22 = -i conj(prb) P; per-image sums
// Ax, Ay, Hxx, Hxy, Hyy; and the horizontal half of S^T: for every object
// column ix, hrow[ix] = sum_tx px(tx -> ix) Y22[tx]  (the vertical half is
// k_casc_vsum; S is separable, so S^T is too).
template <int N, class T>
__global__ void __launch_bounds__(StCfg<N, 3, 1>::THREADS)
k_casc_adj(const float2* __restrict__ tmp, float2* __restrict__ Pc, T* __restrict__ hbuf, const T* __restrict__ c,
           const float* __restrict__ pos, const float* __restrict__ mag, const float2* __restrict__ prb,
           double* __restrict__ rows, CascDims D, const float2* __restrict__ tw4) {
  using CF = StCfg<N, 3, 1>;
  constexpr int TT = CF::T;
  constexpr int E = CF::PL::E;
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(reinterpret_cast<char*>(smem) + CF::FFT_BYTES);
  const int line = threadIdx.x / TT, t = threadIdx.x % TT;
  T* V = reinterpret_cast<T*>(red + red_doubles<TT>(5, CF::THREADS)) +
         (long)line * adj_line_elems(D.nobj, N, (int)sizeof(T));
  const long row = (long)blockIdx.x * CF::LINES + line;
  const bool valid = row < D.nimg * D.nz;
  const long img = valid ? row / D.nz : 0;
  const int ty = valid ? (int)(row % D.nz) : 0;
  const int k = (int)(img % D.ndist);
  const long th = img / D.ndist;
  SmRow sm{smem + line * SmRow::padded(N)};
  const float m0 = valid ? mag[img] : 1.f;
  const float2 r = valid ? ld_pos(pos, img) : make_float2(0.f, 0.f);
  const RowGeo<2> rg(D, m0, r.x, ty);
  if (valid) {
    const float* const w[3] = {rg.py, rg.dpy, rg.d2py};
    vrows_adj<T>(V, V + adj_pair_off(D.nobj), D.nobj, c + coef_off(D, th), rg.yy, w, t, TT);
  }
  dct3_start<N, TT, typename CF::PL>(sm, t, tw4, tmp + row * N, valid);  // ends with a barrier: V is complete
  const T* V0 = V;
  const T* V12 = V + adj_pair_off(D.nobj);
  float s[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  float2 Yr[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int tx = t + i * TT;
    Yr[i] = make_float2(0.f, 0.f);
    if (!valid) continue;
    const float2 G = sm.ld(dct_perm(tx, N));
    const ColGeo<2> cg(D, m0, r.y, tx);
    T x22 = El<T>::zero(), ax = El<T>::zero(), hxx = El<T>::zero();
    T ay = El<T>::zero(), hxy = El<T>::zero(), hyy = El<T>::zero();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const T a0 = V0[cg.xx[j]];
      T a1, a2;
      Pair<T>::ld(V12 + 2 * cg.xx[j], a1, a2);
      El<T>::fma(x22, cg.px[j], a0);
      El<T>::fma(ax, cg.dpx[j], a0);
      El<T>::fma(hxx, cg.d2px[j], a0);
      El<T>::fma(ay, cg.px[j], a1);
      El<T>::fma(hxy, cg.dpx[j], a1);
      El<T>::fma(hyy, cg.px[j], a2);
    }
    const float2 x12 = cexp_i(El<T>::cplx(x22));
    const float2 P = cmulc(G, x12);
    Pc[row * N + tx] = P;
    const float2 pr = prb[((long)k * D.nz + ty) * N + tx];
    // Y22 = -i conj(pr) P  (rec_mpi.py:706-707, .real for float32 objects)
    const T Y = El<T>::proj(rot<false>(cmulc(P, pr)));
    Yr[i] = El<T>::cplx(Y);
    s[0] += El<T>::redot(Y, ax);
    s[1] += El<T>::redot(Y, ay);
    s[2] += El<T>::redot(Y, hxx);
    s[3] += El<T>::redot(Y, hxy);
    s[4] += El<T>::redot(Y, hyy);
  }
  double v[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) v[i] = s[i];
  line_sums<TT, 5>(v, red, line, t);  // contains barriers: G is no longer read
  if (t == 0 && valid) {
#pragma unroll
    for (int i = 0; i < 5; ++i) rows[row * 5 + i] = v[i];  // per-image sums: k_rows_img
  }
  __syncthreads();
  // Y22 into the FFT line; per detector pixel its stencil's first column + 1
  // and tap weights into the gather tables (over V, which is consumed)
  int* tcol = reinterpret_cast<int*>(V);
  float* twt = reinterpret_cast<float*>(tcol + N);
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int tx = t + i * TT;
    sm.st(tx, Yr[i]);
    const float x = sample_x(D, m0, r.y, tx);
    const int ixw = (int)floorf(x);
    float w[4];
    bw0(x - (float)ixw, w);
    tcol[tx] = ixw - 1;
#pragma unroll
    for (int j = 0; j < 4; ++j) twt[j * N + tx] = w[j];
  }
  __syncthreads();
  if (!valid) return;
  const float C0 = -r.y + (m0 - 1.0f) / 2.0f + (float)(D.nobj / 2);
  const float rm0 = cand_rm0(m0);
  T* hrow = hbuf + row * (long)D.nobj;
  for (int ix = t; ix < D.nobj; ix += TT) {
    int lo, hi;
    cand_range_r(rm0, C0, ix, D.n / 2, D.n, lo, hi);
    T acc = El<T>::zero();
    for (int tx = lo; tx <= hi; ++tx) {
      const int j = ix - tcol[tx];  // tap of pixel tx that lands on column ix
      if ((unsigned)j > 3u) continue;
      El<T>::fma(acc, twt[j * N + tx], El<T>::from_sm(sm.ld(tx)));
    }
    hrow[ix] = acc;
  }
}

// ================================================= probe gradient
// gprb[k, p] = sum_theta P[theta, k, p]  (gF1, rec_mpi.py:641)
__global__ void k_sum_theta(const float2* __restrict__ Pc, float2* __restrict__ gprb, long ntheta, int ndist,
                            long npix, float scale, int acc) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // k * npix + p
  if (i >= (long)ndist * npix) return;
  const int k = (int)(i / npix);
  const long p = i % npix;
  double sx = 0.0, sy = 0.0;
  // unrolled: the loads of eight angles are in flight, the sums keep angle order
#pragma unroll 8
  for (long th = 0; th < ntheta; ++th) {
    const float2 v = Pc[(th * ndist + k) * npix + p];
    sx += v.x;
    sy += v.y;
  }
  // the float sum times the variable scaling (rec_mpi.py:345: y[0] * rho_sq['prb'])
  const float2 g = make_float2((float)sx * scale, (float)sy * scale);
  gprb[i] = acc ? cadd(gprb[i], g) : g;   // acc: an angle chunk adds to the earlier chunks' sum
}

// dst[i] += src[i] (the objective and Hessian forms of an angle chunk)
__global__ void k_dacc(double* __restrict__ dst, const double* __restrict__ src, int n) {
  if (threadIdx.x < n) dst[threadIdx.x] += src[threadIdx.x];
}

// ================================================= object gradient
// gc[theta, iy, ix] = sum_k sum_ty py(ty -> iy) hbuf[theta, k, ty, ix]
// (the vertical half of sum_k S_k^T Y22, gF3, rec_mpi.py:802-808).  Each
// thread produces kVRows consecutive rows iy of one column ix, reading each
// detector row that reaches them once (coalesced along ix); every output sums
// its contributions in (k, ty) order.
constexpr int kVRows = 8;

template <class T>
__global__ void __launch_bounds__(256)
k_casc_vsum(T* __restrict__ gc, const T* __restrict__ hbuf, const float* __restrict__ pos,
            const float* __restrict__ mag, CascDims D) {
  const int ix = blockIdx.x * blockDim.x + threadIdx.x;
  const int iy0 = (blockIdx.y * blockDim.y + threadIdx.y) * kVRows;
  const long th = blockIdx.z;
  if (ix >= D.nobj || iy0 >= D.nzobj) return;
  T acc[kVRows];
#pragma unroll
  for (int r = 0; r < kVRows; ++r) acc[r] = El<T>::zero();
  for (int k = 0; k < D.ndist; ++k) {
    const long img = th * D.ndist + k;
    const float m0 = mag[img];
    const float ry = pos[2 * img + 0];
    const float C0 = -ry + (m0 - 1.0f) / 2.0f + (float)(D.nzobj / 2);
    int a0, a1, b0, b1;
    cand_range(m0, C0, iy0, D.nz / 2, D.nz, a0, a1);
    cand_range(m0, C0, min(iy0 + kVRows - 1, D.nzobj - 1), D.nz / 2, D.nz, b0, b1);
    const int ty0 = min(a0, b0), ty1 = max(a1, b1);
    const T* hb = hbuf + img * (long)D.nz * D.nobj + ix;
    for (int ty = ty0; ty <= ty1; ++ty) {
      const float y = sample_y(D, m0, ry, ty);
      const int iyw = (int)floorf(y);
      const int jr = iy0 - iyw + 1;          // tap index of row iy0
      if (jr > 3 || jr + kVRows - 1 < 0) continue;
      float w[4];
      bw0(y - (float)iyw, w);
      const T h = __ldg(&hb[(long)ty * D.nobj]);
#pragma unroll
      for (int r = 0; r < kVRows; ++r) {
        const int j = jr + r;
        const float wt = (j == 0) ? w[0] : (j == 1) ? w[1] : (j == 2) ? w[2] : (j == 3) ? w[3] : 0.f;
        if (j >= 0 && j <= 3) El<T>::fma(acc[r], wt, h);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kVRows; ++r)
    if (iy0 + r < D.nzobj) gc[(th * D.nzobj + iy0 + r) * D.nobj + ix] = acc[r];
}

// gpos[img] = (-Ay, -Ax)  (dsadj, cuda_kernels.py:744-761 with redot)
// times the variable scaling (rec_mpi.py:347: y[2] * rho_sq['pos'])
__global__ void k_casc_gpos(const double* __restrict__ acc_img, float* __restrict__ gpos, long nimg, float scale) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nimg) return;
  gpos[2 * i + 0] = (float)(-acc_img[i * kNAcc + kAy]) * scale;
  gpos[2 * i + 1] = (float)(-acc_img[i * kNAcc + kAx]) * scale;
}

// ================================================ Hessian row pass
// For NDIR directions d: y22_d = dS(c, c_d, r_d);  v_d = x12 (prb_d + i prb y22_d)
// -> row DCT-II -> tmp[d];  plus the pointwise second-order sums L1, L2
// (pairs 00, 01, 11) and the per-image Ax(c_d), Ay(c_d).
template <int N, class T, int NDIR>
__global__ void __launch_bounds__(StCfg<N, 2 * (1 + NDIR), NDIR>::THREADS)
k_casc_hess_fwd(const T* __restrict__ c, const float* __restrict__ pos, const float* __restrict__ mag,
                const float2* __restrict__ prb, const float2* __restrict__ Pc, const T* __restrict__ c0,
                const float* __restrict__ pos0, const float2* __restrict__ prb0, const T* __restrict__ c1,
                const float* __restrict__ pos1, const float2* __restrict__ prb1, float2* __restrict__ tmp,
                double* __restrict__ rows, CascDims D,
                const float2* __restrict__ tw4) {
  constexpr int NS = 2 * (1 + NDIR);
  using CF = StCfg<N, NS, NDIR>;
  constexpr int TT = CF::TR;  // threads of a detector row; CF::T of them per FFT line
  constexpr int LINES = CF::LINES;
  constexpr int K = (NDIR == 2) ? 10 : 4;
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(reinterpret_cast<char*>(smem) + CF::FFT_BYTES);
  const int line = threadIdx.x / TT, t = threadIdx.x % TT;
  T* V = reinterpret_cast<T*>(red + red_doubles<TT>(K, CF::THREADS)) + (long)line * NS * D.nobj;
  const long row = (long)blockIdx.x * LINES + line;
  const bool valid = row < D.nimg * D.nz;
  const long img = valid ? row / D.nz : 0;
  const int ty = valid ? (int)(row % D.nz) : 0;
  const int k = (int)(img % D.ndist);
  const long th = img / D.ndist;
  SmRow sm0{smem + line * SmRow::padded(N)};
  SmRow sm1{smem + (LINES + line) * SmRow::padded(N)};
  const long coff = coef_off(D, th);
  const float m0 = valid ? mag[img] : 1.f;
  const float2 r = valid ? ld_pos(pos, img) : make_float2(0.f, 0.f);
  const float2 rd0 = valid ? ld_pos(pos0, img) : make_float2(0.f, 0.f);
  const float2 rd1 = (valid && NDIR == 2) ? ld_pos(pos1, img) : make_float2(0.f, 0.f);
  // P streams from DRAM: each pixel's value is loaded one pixel ahead (the
  // first before the vertical pass), so its latency overlaps other work
  const float2* Prow = Pc + row * N;
  float2 Pnext = valid ? Prow[t] : make_float2(0.f, 0.f);
  {
    const RowGeo<1> rg(D, m0, r.x, ty);
    if (valid) {
      const float* const w[2] = {rg.py, rg.dpy};
      // sets, interleaved per object column (V[ix * NS + set]):
      // (c, py) (c, dpy) (c_y, py) (c_y, dpy) [(c_z, py) (c_z, dpy)]
      vrows_pair<T, NS>(V, 0, D.nobj, c + coff, rg.yy, w[0], w[1], t, TT);
      vrows_pair<T, NS>(V, 2, D.nobj, c0 + coff, rg.yy, w[0], w[1], t, TT);
      if (NDIR == 2) vrows_pair<T, NS>(V, 4, D.nobj, c1 + coff, rg.yy, w[0], w[1], t, TT);
    }
  }
  __syncthreads();
  // sums: L1 00,01,11 ; L2 00,01,11 ; A: ax0, ay0, ax1, ay1
  float s[10] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  for (int tx = t; tx < N; tx += TT) {
    float2 v0 = make_float2(0.f, 0.f), v1 = make_float2(0.f, 0.f);
    const float2 P = Pnext;
    if (valid && tx + TT < N) Pnext = Prow[tx + TT];
    if (valid) {
      const ColGeo<1> cg(D, m0, r.y, tx);
      // the horizontal taps: every set of one tap's column in NS / 2 vector loads
      T x22 = El<T>::zero(), dxc = El<T>::zero(), dyc = El<T>::zero();
      T s0 = El<T>::zero(), ax0 = El<T>::zero(), ay0 = El<T>::zero();
      T s1 = El<T>::zero(), ax1 = El<T>::zero(), ay1 = El<T>::zero();
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const T* col = V + (long)cg.xx[j] * NS;
        T a0, a1, a2, a3;
        Pair<T>::ld(col, a0, a1);
        Pair<T>::ld(col + 2, a2, a3);
        El<T>::fma(x22, cg.px[j], a0);
        El<T>::fma(dxc, cg.dpx[j], a0);
        El<T>::fma(dyc, cg.px[j], a1);
        El<T>::fma(s0, cg.px[j], a2);
        El<T>::fma(ax0, cg.dpx[j], a2);
        El<T>::fma(ay0, cg.px[j], a3);
        if (NDIR == 2) {
          T a4, a5;
          Pair<T>::ld(col + 4, a4, a5);
          El<T>::fma(s1, cg.px[j], a4);
          El<T>::fma(ax1, cg.dpx[j], a4);
          El<T>::fma(ay1, cg.px[j], a5);
        }
      }
      // dS (rec_mpi.py:757; cuda_kernels.py:600-609): sum phi phi c_d - (dphi_x phi_y r_dx + phi_x dphi_y r_dy) c
      T y0 = s0, y1 = s1;
      El<T>::fma(y0, -rd0.y, dxc);
      El<T>::fma(y0, -rd0.x, dyc);
      if (NDIR == 2) {
        El<T>::fma(y1, -rd1.y, dxc);
        El<T>::fma(y1, -rd1.x, dyc);
      }
      const float2 x12 = cexp_i(El<T>::cplx(x22));
      const long p = ((long)k * D.nz + ty) * N + tx;
      const float2 pr = prb[p];
      const T Y = El<T>::proj(rot<false>(cmulc(P, pr)));
      const float2 Y0 = El<T>::cplx(y0), Y1 = El<T>::cplx(y1);
      const float2 q0 = prb0[p];
      const float2 q1 = (NDIR == 2) ? prb1[p] : make_float2(0.f, 0.f);
      // v_d = x12 (prb_d + i prb y22_d)   (dF2 then dF1, rec_mpi.py:591, 664)
      v0 = cmul(x12, cadd(q0, cmul_i(cmul(pr, Y0))));
      if (NDIR == 2) v1 = cmul(x12, cadd(q1, cmul_i(cmul(pr, Y1))));
      // L1(a,b) = Re(conj(P) i (q_a y22_b + q_b y22_a));  L2(a,b) = -Re(conj(P) prb y22_a y22_b),
      // with the factors the forms share formed once: u_d = i conj(P) q_d, A = conj(P) prb
      const float2 cP = cconj(P);
      const float2 iP = cmul_i(cP);
      const float2 u0 = cmul(iP, q0);
      const float2 A = cmul(cP, pr);
      const float2 a0 = cmul(A, Y0);
      auto re = [](float2 x, float2 y) { return x.x * y.x - x.y * y.y; };  // Re(x y)
      s[0] += 2.f * re(u0, Y0);
      s[3] -= re(a0, Y0);
      s[6] += El<T>::redot(Y, ax0);
      s[7] += El<T>::redot(Y, ay0);
      if (NDIR == 2) {
        const float2 u1 = cmul(iP, q1);
        s[1] += re(u0, Y1) + re(u1, Y0);
        s[2] += 2.f * re(u1, Y1);
        s[4] -= re(a0, Y1);
        s[5] -= re(cmul(A, Y1), Y1);
        s[8] += El<T>::redot(Y, ax1);
        s[9] += El<T>::redot(Y, ay1);
      }
    }
    dct2_put<N>(sm0, tx, v0);
    if (NDIR == 2) dct2_put<N>(sm1, tx, v1);
  }
  double v[K];
  if (NDIR == 2) {
#pragma unroll
    for (int i = 0; i < K; ++i) v[i] = s[i];
  } else {
    v[0] = s[0];
    v[1] = s[3];
    v[2] = s[6];
    v[3] = s[7];
  }
  line_sums<TT, K>(v, red, line, t);
  // per-row sums in the slots L1 00,01,11, L2 00,01,11, Ayx, Ayy, Azx, Azy
  // (reduced by k_rows_img / k_imgs_glob)
  if (t == 0 && valid) {
    double* rw = rows + row * kHessRowK;
    if (NDIR == 2) {
#pragma unroll
      for (int i = 0; i < K; ++i) rw[i] = v[i];
    } else {
      rw[0] = v[0];
      rw[3] = v[1];
      rw[6] = v[2];
      rw[7] = v[3];
      rw[1] = rw[2] = rw[4] = rw[5] = rw[8] = rw[9] = 0.0;
    }
  }
  __syncthreads();
  // direction d's line is transformed by the row's d-th group of CF::T threads
  const long nrow = D.nimg * D.nz;
  const int d = t / CF::T;
  dct2_finish<N, CF::T, typename CF::PL>(d == 0 ? sm0 : sm1, t % CF::T, tw4, tmp + (d * nrow + row) * N, valid);
}

// ======================================== Hessian quadratic terms
// y0_d = DCT-III rows of tmp[d];  Q pairs with x0 and the data.
template <int N, int NDIR>
__global__ void __launch_bounds__(RowCfg<N>::THREADS, 3)
k_casc_hess_q(const float2* __restrict__ tmp, const float2* __restrict__ x0c, const float* __restrict__ data,
              double* __restrict__ rows, CascDims D, const float2* __restrict__ tw4) {
  constexpr int TT = RowCfg<N>::T;
  constexpr int LINES = RowCfg<N>::LINES;
  extern __shared__ float2 smem[];
  double* red = reinterpret_cast<double*>(smem + NDIR * LINES * SmRow::padded(N));
  const int line = threadIdx.x / TT, t = threadIdx.x % TT;
  const long row = (long)blockIdx.x * LINES + line;
  const bool valid = row < D.nimg * D.nz;
  const long nrow = D.nimg * D.nz;
  SmRow sm0{smem + line * SmRow::padded(N)};
  SmRow sm1{smem + (LINES + line) * SmRow::padded(N)};
  constexpr int E = Plan<N>::E;
  dct3_start<N, TT>(sm0, t, tw4, tmp + row * N, valid);
  if (NDIR == 2) dct3_start<N, TT>(sm1, t, tw4, tmp + (nrow + row) * N, valid);
  float s[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int tx = t + i * TT;
    if (!valid) break;
    const float2 x0 = x0c[row * N + tx];
    const float d = data[row * N + tx];
    const float a = sqrtf(x0.x * x0.x + x0.y * x0.y);
    const float2 l0 = make_float2(x0.x / a, x0.y / a);
    const float d0 = d / a;
    const float2 y0 = sm0.ld(dct_perm(tx, N));
    const float ly = l0.x * y0.x + l0.y * y0.y;  // Re(conj(l0) y0)
    s[0] += (1.f - d0) * (y0.x * y0.x + y0.y * y0.y) + d0 * ly * ly;
    if (NDIR == 2) {
      const float2 y1 = sm1.ld(dct_perm(tx, N));
      const float lz = l0.x * y1.x + l0.y * y1.y;
      s[1] += (1.f - d0) * (y0.x * y1.x + y0.y * y1.y) + d0 * ly * lz;
      s[2] += (1.f - d0) * (y1.x * y1.x + y1.y * y1.y) + d0 * lz * lz;
    }
  }
  double v[3] = {s[0], s[1], s[2]};
  line_sums<TT, 3>(v, red, line, t);
  if (t == 0 && valid) {
#pragma unroll
    for (int i = 0; i < 3; ++i) rows[row * 3 + i] = v[i];  // Q0, Q1, Q2: k_rows_img / k_imgs_glob
  }
}

// ============================================ row sums -> image / total sums
// The row kernels write each detector row's sums (FP64, reduced over the
// row's threads) to rows [nimg * nz][K]; these two kernels add them up in a
// fixed order, so the sums do not depend on scheduling and no two rows
// contend for one accumulator.

// imgs[img][i] = sum over the image's nz rows of rows[.][i] (one block per
// image); the slots i0 .. i0 + na - 1 are also added to acc_img[img][a0 + .].
__global__ void __launch_bounds__(kRedThreads)
k_rows_img(const double* __restrict__ rows, int K, int nz, double* __restrict__ imgs, double* __restrict__ acc_img,
           int a0, int i0, int na) {
  const long img = blockIdx.x;
  __shared__ double red[kRowKMax][kRedThreads / 32];
  double s[kRowKMax];
#pragma unroll
  for (int i = 0; i < kRowKMax; ++i) s[i] = 0.0;
  for (int ty = threadIdx.x; ty < nz; ty += kRedThreads) {
    const double* rw = rows + (img * nz + ty) * K;
#pragma unroll
    for (int i = 0; i < kRowKMax; ++i)
      if (i < K) s[i] += rw[i];
  }
#pragma unroll
  for (int i = 0; i < kRowKMax; ++i) {
    if (i >= K) break;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[i] += __shfl_down_sync(0xffffffffu, s[i], o);
    if ((threadIdx.x & 31) == 0) red[i][threadIdx.x / 32] = s[i];
  }
  __syncthreads();
  if (threadIdx.x < K) {
    const int i = threadIdx.x;
    double tot = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) tot += red[i][w];
    imgs[img * K + i] = tot;
    if (i >= i0 && i < i0 + na) acc_img[img * kNAcc + a0 + (i - i0)] += tot;
  }
}

// glob[g0 + i] += sum over images of imgs[img][i]  (block i)
__global__ void __launch_bounds__(kRedThreads)
k_imgs_glob(const double* __restrict__ imgs, int K, long nimg, double* __restrict__ glob, int g0) {
  const int i = blockIdx.x;
  __shared__ double red[kRedThreads / 32];
  double s = 0.0;
  for (long img = threadIdx.x; img < nimg; img += kRedThreads) s += imgs[img * K + i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x / 32] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < kRedThreads / 32; ++w) tot += red[w];
    glob[g0 + i] += tot;
  }
}

// ============================================ Hessian combination
// out[0] = H(y,y), out[1] = H_ref(y,z), out[2] = H(z,z), out[3] = H_sym(y,z)
__global__ void k_casc_hess_combine(const double* __restrict__ acc_img, const double* __restrict__ glob,
                                    const float* __restrict__ posy, const float* __restrict__ posz, int ndir,
                                    long nimg, double qscale, int acc, double* __restrict__ out) {
  double b00 = 0, b01 = 0, b11 = 0, ayy = 0, azz = 0, ayz = 0, azy = 0;
  for (long i = threadIdx.x; i < nimg; i += blockDim.x) {
    const double* a = acc_img + i * kNAcc;
    const double yx = posy[2 * i + 1], yy = posy[2 * i + 0];
    b00 += yx * yx * a[kHxx] + 2.0 * yx * yy * a[kHxy] + yy * yy * a[kHyy];
    ayy += -(yx * a[kAyx] + yy * a[kAyy]);
    if (ndir == 2) {
      const double zx = posz[2 * i + 1], zy = posz[2 * i + 0];
      b01 += yx * zx * a[kHxx] + (yx * zy + yy * zx) * a[kHxy] + yy * zy * a[kHyy];
      b11 += zx * zx * a[kHxx] + 2.0 * zx * zy * a[kHxy] + zy * zy * a[kHyy];
      azz += -(zx * a[kAzx] + zy * a[kAzy]);
      ayz += -(zx * a[kAyx] + zy * a[kAyy]);  // c_y with r_z
      azy += -(yx * a[kAzx] + yy * a[kAzy]);  // c_z with r_y
    }
  }
  __shared__ double red[7][256];
  double vals[7] = {b00, b01, b11, ayy, azz, ayz, azy};
  for (int j = 0; j < 7; ++j) red[j][threadIdx.x] = vals[j];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int j = 0; j < 7; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    b00 = red[0][0];
    b01 = red[1][0];
    b11 = red[2][0];
    ayy = red[3][0];
    azz = red[4][0];
    ayz = red[5][0];
    azy = red[6][0];
    double h[4] = {qscale * glob[kQ0] + glob[kL10] + glob[kL20] + b00 + 2.0 * ayy, 0.0, 0.0, 0.0};
    if (ndir == 2) {
      const double common = qscale * glob[kQ1] + glob[kL11] + glob[kL21] + b01;
      h[1] = common + ayy + azz;
      h[2] = qscale * glob[kQ2] + glob[kL12] + glob[kL22] + b11 + 2.0 * azz;
      h[3] = common + ayz + azy;
    }
    for (int i = 0; i < 4; ++i) out[i] = acc ? out[i] + h[i] : h[i];   // acc: an angle chunk
  }
}

}  // namespace ht

#define HT_REC_SIZES(X) X(32) X(64) X(128) X(256) X(384) X(512) X(768) X(1024) X(2048)

// ================================================================= C ABI
struct ht_rec_s {
  ht::CascDims D;
  int ntheta, is_complex, device;
  const ht_prop_s* prop;
  float2* x0;      // [nimg, nz, n]
  float2* P;       // [nimg, nz, n]
  float2* tmp;     // [2, nimg, nz, n]
  double* acc_img; // [nimg, kNAcc]
  double* glob;    // [kNGlob]
  double* rows;    // [nimg * nz, kRowKMax] per-row sums of the row kernels
  double* imgs;    // [nimg, kRowKMax] their per-image sums
  double ndata;    // N of the objective's 2/N: ntheta*ndist*nz*n, or the whole problem's for an angle chunk
};

extern "C" int ht_rec_create(int n, int nz, int nobj, int nzobj, int ntheta, int ndist, int is_complex,
                             ht_prop_s* prop, ht_rec_s** out) {
  using namespace ht;
  HT_REQUIRE(out && prop, "ht_rec_create: null pointer");
  HT_REQUIRE(n > 0 && nz > 0 && nobj > 0 && nzobj > 0 && ntheta > 0 && ndist > 0, "ht_rec_create: bad sizes");
  int pn, pnz, pnd;
  prop_dims(prop, &pn, &pnz, &pnd);
  HT_REQUIRE(pn == n && pnz == nz && pnd == ndist, "ht_rec_create: propagator sizes differ");
  bool n_ok = false;
#define X(S) n_ok = n_ok || (n == S);
  HT_REC_SIZES(X)
#undef X
  if (!n_ok) {
    set_error("ht_rec_create: n must be one of 32, 64, 128, 256, 384, 512, 768, 1024, 2048");
    return kUnsupported;
  }
  ht_rec_s* r = new ht_rec_s{};
  r->D = CascDims{n, nz, nobj, nzobj, ndist, (long)ntheta * ndist};
  r->ntheta = ntheta;
  r->ndata = (double)ntheta * ndist * nz * n;
  r->is_complex = is_complex ? 1 : 0;
  r->prop = prop;
  cudaGetDevice(&r->device);
  const size_t img = (size_t)ntheta * ndist * nz * n;
  cudaError_t e = cudaMalloc(&r->x0, sizeof(float2) * img);
  if (e == cudaSuccess) e = cudaMalloc(&r->P, sizeof(float2) * img);
  // tmp: two spectra for the Hessian pass; during the gradient pass its
  // second part holds the horizontal S^T rows [nimg, nz, nobj] of T
  const size_t hrow = ((size_t)ntheta * ndist * nz * nobj * (is_complex ? 8 : 4) + 7) / 8;
  if (e == cudaSuccess) e = cudaMalloc(&r->tmp, sizeof(float2) * (img + std::max(img, hrow)));
  if (e == cudaSuccess) e = cudaMalloc(&r->acc_img, sizeof(double) * (size_t)ntheta * ndist * kNAcc);
  if (e == cudaSuccess) e = cudaMalloc(&r->glob, sizeof(double) * kNGlob);
  if (e == cudaSuccess) e = cudaMalloc(&r->rows, sizeof(double) * (size_t)ntheta * ndist * nz * kRowKMax);
  if (e == cudaSuccess) e = cudaMalloc(&r->imgs, sizeof(double) * (size_t)ntheta * ndist * kRowKMax);
  if (e != cudaSuccess) {
    set_error(std::string("ht_rec_create: ") + cudaGetErrorString(e));
    cudaFree(r->x0);
    cudaFree(r->P);
    cudaFree(r->tmp);
    cudaFree(r->acc_img);
    cudaFree(r->glob);
    cudaFree(r->rows);
    cudaFree(r->imgs);
    delete r;
    return kCudaError;
  }
  *out = r;
  return kOk;
}

extern "C" int ht_rec_destroy(ht_rec_s* r) {
  if (!r) return ht::kOk;
  cudaFree(r->x0);
  cudaFree(r->P);
  cudaFree(r->tmp);
  cudaFree(r->acc_img);
  cudaFree(r->glob);
  cudaFree(r->rows);
  cudaFree(r->imgs);
  delete r;
  return ht::kOk;
}

namespace ht {
#define HT_ROWS_GRID(N, nrows) (unsigned)(((nrows) + RowCfg<N>::LINES - 1) / RowCfg<N>::LINES)

// Dynamic shared memory of the stencil row kernels, checked against the device
// limit (the vertically reduced rows grow with nobj).
template <class CF>
static cudaError_t stencil_smem(const void* kernel, int K, int nobj, int elem, int* bytes) {
  *bytes = CF::bytes(K, nobj, elem);
  if (*bytes > 227 * 1024) {
    set_error("fused cascade: nobj = " + std::to_string(nobj) + " needs " + std::to_string(*bytes) +
              " bytes of shared memory per block (limit 227 KB)");
    return cudaErrorInvalidValue;
  }
  return cudaSuccess;
}

// Sum the per-row values a row kernel left in r->rows (K a row): per image
// into r->imgs (slots i0.. i0+na-1 also into acc_img[.][a0..]), and slots
// 0..ng-1 over all images into glob[g0..].
static cudaError_t reduce_rows(ht_rec_s* r, int K, int a0, int i0, int na, int g0, int ng, cudaStream_t st) {
  k_rows_img<<<(unsigned)r->D.nimg, kRedThreads, 0, st>>>(r->rows, K, r->D.nz, r->imgs, r->acc_img, a0, i0, na);
  ::ht::count_launch();
  if (ng > 0) {
    k_imgs_glob<<<(unsigned)ng, kRedThreads, 0, st>>>(r->imgs, K, r->D.nimg, r->glob, g0);
    ::ht::count_launch();
  }
  return cudaGetLastError();
}

template <int N, class T>
static cudaError_t launch_fwd(const CascDims& D, const T* c, const float* pos, const float* mag, const float2* prb,
                              float2* tmp, const float2* twn, cudaStream_t st) {
  using CF = StCfg<N, 1, 1>;
  int smem = 0;
  cudaError_t e = stencil_smem<CF>(nullptr, 0, D.nobj, (int)sizeof(T), &smem);
  if (e == cudaSuccess) e = allow_smem(k_casc_fwd<N, T>, smem);
  if (e != cudaSuccess) return e;
  const long nrows = D.nimg * D.nz;
  {
    KTimer kt("k_casc_fwd", st, (double)D.nimg);
    k_casc_fwd<N, T><<<(unsigned)((nrows + CF::LINES - 1) / CF::LINES), CF::THREADS, smem, st>>>(c, pos, mag, prb,
                                                                                               tmp, D, twn);
  }
  ::ht::count_launch();
  return cudaGetLastError();
}

template <int N, class T>
static cudaError_t fwd_pass(ht_rec_s* r, const void* c, const float* pos, const float* mag, const float2* prb,
                            const float2* hw, const float2* twn, const float2* twz, cudaStream_t st) {
  cudaError_t e = launch_fwd<N, T>(r->D, (const T*)c, pos, mag, prb, r->tmp, twn, st);
  if (e != cudaSuccess) return e;
  return dct_cols(r->D.nz, false, r->tmp, r->D.nimg, N, hw, r->D.ndist, twz, st);
}

template <int N, int MODE>
static cudaError_t resid_pass(ht_rec_s* r, const float* data, float* amp, float scale, const float2* twn,
                              cudaStream_t st) {
  using CF = RowCfg<N>;
  const int smem = CF::SMEM + red_doubles<CF::T>(1, CF::THREADS) * (int)sizeof(double);
  cudaError_t e = allow_smem(k_casc_resid<N, MODE>, smem);
  if (e != cudaSuccess) return e;
  const long nrows = r->D.nimg * r->D.nz;
  if constexpr (N == kR512) {
    KTimer kt(MODE == 0 ? "k_casc_resid" : "k_casc_resid_f", st, (double)r->D.nimg);
    k_casc_resid512<MODE><<<(unsigned)((nrows + kR512Lines - 1) / kR512Lines), 32 * kR512Lines, 0, st>>>(
        r->tmp, r->x0, data, amp, r->glob, MODE == 2 ? nullptr : r->rows, scale, r->D, twn);
  } else {
    KTimer kt(MODE == 0 ? "k_casc_resid" : "k_casc_resid_f", st, (double)r->D.nimg);
    k_casc_resid<N, MODE><<<HT_ROWS_GRID(N, nrows), CF::THREADS, smem, st>>>(
        r->tmp, r->x0, data, amp, r->glob, MODE == 2 ? nullptr : r->rows, scale, r->D, twn);
  }
  ::ht::count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return MODE == 2 ? cudaSuccess : reduce_rows(r, 1, 0, 0, 0, kF, 1, st);
}

template <int N, class T>
static cudaError_t grad_impl(ht_rec_s* r, const void* c, const float* pos, const float* mag, const float2* prb,
                             const float* data, void* gc, float* gpos, float2* gprb, float scale, float spos,
                             float sprb, int acc, cudaStream_t st) {
  const float2 *hw, *twn, *twz;
  prop_tables(r->prop, &hw, &twn, &twz);
  cudaError_t e = fwd_pass<N, T>(r, c, pos, mag, prb, hw, twn, twz, st);
  if (e != cudaSuccess) return e;
  if ((e = resid_pass<N, 0>(r, data, nullptr, scale, twn, st)) != cudaSuccess) return e;
  if ((e = dct_cols(r->D.nz, true, r->tmp, r->D.nimg, N, hw, r->D.ndist, twz, st)) != cudaSuccess) return e;
  using CA = StCfg<N, 3, 1>;
  const long nrows = r->D.nimg * r->D.nz;
  const int smem = CA::FFT_BYTES + red_doubles<CA::TR>(5, CA::THREADS) * (int)sizeof(double) +
                   CA::LINES * adj_line_elems(r->D.nobj, N, (int)sizeof(T)) * (int)sizeof(T);
  if (smem > 227 * 1024) {
    set_error("fused cascade: nobj = " + std::to_string(r->D.nobj) + " needs " + std::to_string(smem) +
              " bytes of shared memory per block (limit 227 KB)");
    return cudaErrorInvalidValue;
  }
  if ((e = allow_smem(k_casc_adj<N, T>, smem)) != cudaSuccess) return e;
  T* hbuf = reinterpret_cast<T*>(r->tmp + nrows * N);
  {
    KTimer kt("k_casc_adj", st, (double)r->D.nimg);
    k_casc_adj<N, T><<<(unsigned)((nrows + CA::LINES - 1) / CA::LINES), CA::THREADS, smem, st>>>(
        r->tmp, r->P, hbuf, (const T*)c, pos, mag, prb, r->rows, r->D, twn);
  }
  ::ht::count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = reduce_rows(r, 5, kAx, 0, 5, 0, 0, st)) != cudaSuccess) return e;
  const long npix = (long)r->D.nz * N;
  k_sum_theta<<<(unsigned)((r->D.ndist * npix + 255) / 256), 256, 0, st>>>(r->P, gprb, r->ntheta, r->D.ndist, npix,
                                                                             sprb, acc);
  ::ht::count_launch();
  if (r->D.shared_c) {
    // one coefficient array for all angles: its gradient sums every image
    // (all images taken as the distances of a single angle)
    CascDims all = r->D;
    all.ndist = (int)r->D.nimg;
    dim3 g1((r->D.nobj + 31) / 32, (r->D.nzobj + 8 * kVRows - 1) / (8 * kVRows), 1);
    k_casc_vsum<T><<<g1, dim3(32, 8), 0, st>>>((T*)gc, hbuf, pos, mag, all);
  } else {
    dim3 g2((r->D.nobj + 31) / 32, (r->D.nzobj + 8 * kVRows - 1) / (8 * kVRows), r->ntheta);
    k_casc_vsum<T><<<g2, dim3(32, 8), 0, st>>>((T*)gc, hbuf, pos, mag, r->D);
  }
  ::ht::count_launch();
  k_casc_gpos<<<(unsigned)((r->D.nimg + 255) / 256), 256, 0, st>>>(r->acc_img, gpos, r->D.nimg, spos);
  ::ht::count_launch();
  return cudaGetLastError();
}

template <int N, class T, int NDIR>
static cudaError_t hess_impl(ht_rec_s* r, const void* c, const float* pos, const float* mag, const float2* prb,
                             const float* data, const void* c0, const float* p0, const float2* q0, const void* c1,
                             const float* p1, const float2* q1, cudaStream_t st) {
  const float2 *hw, *twn, *twz;
  prop_tables(r->prop, &hw, &twn, &twz);
  using CF = RowCfg<N>;
  using CH = StCfg<N, 2 * (1 + NDIR), NDIR>;
  const long nrows = r->D.nimg * r->D.nz;
  int smem = 0;
  cudaError_t e = stencil_smem<CH>(nullptr, NDIR == 2 ? 10 : 4, r->D.nobj, (int)sizeof(T), &smem);
  if (e == cudaSuccess) e = allow_smem(k_casc_hess_fwd<N, T, NDIR>, smem);
  if (e != cudaSuccess) return e;
  {
    KTimer kt("k_casc_hess_fwd", st, (double)NDIR * r->D.nimg);
    k_casc_hess_fwd<N, T, NDIR><<<(unsigned)((nrows + CH::LINES - 1) / CH::LINES), CH::THREADS, smem, st>>>(
        (const T*)c, pos, mag, prb, r->P, (const T*)c0, p0, q0, (const T*)c1, p1, q1, r->tmp, r->rows,
        r->D, twn);
  }
  ::ht::count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // rows slots 0-5: L1/L2 sums (glob kL10..kL22); 6-9: Ayx, Ayy, Azx, Azy (acc_img)
  if ((e = reduce_rows(r, kHessRowK, kAyx, 6, 4, kL10, 6, st)) != cudaSuccess) return e;
  if ((e = dct_cols(r->D.nz, false, r->tmp, NDIR * r->D.nimg, N, hw, r->D.ndist, twz, st)) != cudaSuccess) return e;
  const int smq = NDIR * CF::SMEM + red_doubles<CF::T>(3, CF::THREADS) * (int)sizeof(double);
  if ((e = allow_smem(k_casc_hess_q<N, NDIR>, smq)) != cudaSuccess) return e;
  if constexpr (N == kR512) {
    KTimer kt("k_casc_hess_q", st, (double)NDIR * r->D.nimg);
    k_casc_hess_q512<NDIR><<<(unsigned)((nrows + kR512Lines - 1) / kR512Lines), 32 * kR512Lines, 0, st>>>(
        r->tmp, r->x0, data, r->rows, r->D, twn);
  } else {
    KTimer kt("k_casc_hess_q", st, (double)NDIR * r->D.nimg);
    k_casc_hess_q<N, NDIR><<<HT_ROWS_GRID(N, nrows), CF::THREADS, smq, st>>>(r->tmp, r->x0, data, r->rows, r->D,
                                                                             twn);
  }
  ::ht::count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  return reduce_rows(r, 3, 0, 0, 0, kQ0, 3, st);
}


}  // namespace ht

extern "C" int ht_rec_forward(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb,
                              const float* data, float* amp, double* fval, void* stream) {
  using namespace ht;
  HT_REQUIRE(r && c && pos && mag && prb, "ht_rec_forward: null pointer");
  HT_REQUIRE(amp || (data && fval), "ht_rec_forward: need data and fval, or amp");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float2 *hw, *twn, *twz;
  prop_tables(r->prop, &hw, &twn, &twz);
  HT_CHECK_CUDA(cudaMemsetAsync(r->glob, 0, sizeof(double) * kNGlob, st));
  cudaError_t e = cudaErrorInvalidValue;
  switch (r->D.n) {
#define X(S)                                                                                                  \
  case S:                                                                                                     \
    e = r->is_complex ? fwd_pass<S, float2>(r, c, pos, mag, (const float2*)prb, hw, twn, twz, st)              \
                      : fwd_pass<S, float>(r, c, pos, mag, (const float2*)prb, hw, twn, twz, st);              \
    if (e == cudaSuccess)                                                                                     \
      e = amp ? resid_pass<S, 2>(r, data, amp, 0.f, twn, st) : resid_pass<S, 1>(r, data, nullptr, 0.f, twn, st); \
    break;
    HT_REC_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  if (fval) HT_CHECK_CUDA(cudaMemcpyAsync(fval, r->glob + kF, sizeof(double), cudaMemcpyDeviceToDevice, st));
  return kOk;
}

extern "C" int ht_rec_set_shared_coefficients(ht_rec_s* r, int shared) {
  using namespace ht;
  HT_REQUIRE(r, "ht_rec_set_shared_coefficients: null pointer");
  r->D.shared_c = shared ? 1 : 0;
  return kOk;
}

extern "C" int ht_rec_set_data_size(ht_rec_s* r, double ndata) {
  using namespace ht;
  HT_REQUIRE(r, "ht_rec_set_data_size: null pointer");
  HT_REQUIRE(ndata >= (double)r->ntheta * r->D.ndist * r->D.nz * r->D.n,
             "ht_rec_set_data_size: N is smaller than the handle's own ntheta*ndist*nz*n");
  r->ndata = ndata;
  return kOk;
}

extern "C" int ht_rec_gradient(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb,
                               const float* data, void* gc, float* gpos, void* gprb, double* fval, float scale_pos,
                               float scale_prb, int accumulate, void* stream) {
  using namespace ht;
  HT_REQUIRE(r && c && pos && mag && prb && data && gc && gpos && gprb, "ht_rec_gradient: null pointer");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HT_CHECK_CUDA(cudaMemsetAsync(r->glob, 0, sizeof(double) * kNGlob, st));
  HT_CHECK_CUDA(cudaMemsetAsync(r->acc_img, 0, sizeof(double) * r->D.nimg * kNAcc, st));
  // rec_mpi.py:569: np.float32(2 / data_size)
  const float scale = (float)(2.0 / r->ndata);
  cudaError_t e = cudaErrorInvalidValue;
  switch (r->D.n) {
#define X(S)                                                                                                     \
  case S:                                                                                                        \
    e = r->is_complex ? grad_impl<S, float2>(r, c, pos, mag, (const float2*)prb, data, gc, gpos, (float2*)gprb,    \
                                             scale, scale_pos, scale_prb, accumulate, st)                        \
                      : grad_impl<S, float>(r, c, pos, mag, (const float2*)prb, data, gc, gpos, (float2*)gprb,     \
                                            scale, scale_pos, scale_prb, accumulate, st);                        \
    break;
    HT_REC_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  if (fval && accumulate) {
    k_dacc<<<1, 32, 0, st>>>(fval, r->glob + kF, 1);
    ::ht::count_launch();
    HT_CHECK_CUDA(cudaGetLastError());
  } else if (fval) {
    HT_CHECK_CUDA(cudaMemcpyAsync(fval, r->glob + kF, sizeof(double), cudaMemcpyDeviceToDevice, st));
  }
  return kOk;
}

extern "C" int ht_rec_hessian(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb,
                              const float* data, int ndir, const void* cy, const float* posy, const void* prby,
                              const void* cz, const float* posz, const void* prbz, double* out, int accumulate,
                              void* stream) {
  using namespace ht;
  HT_REQUIRE(r && c && pos && mag && prb && data && cy && posy && prby && out, "ht_rec_hessian: null pointer");
  HT_REQUIRE(ndir == 1 || (ndir == 2 && cz && posz && prbz), "ht_rec_hessian: ndir must be 1, or 2 with z given");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // clear the Hessian slots only: the gradient pass's per-image terms stay
  HT_CHECK_CUDA(cudaMemsetAsync(r->glob + kQ0, 0, sizeof(double) * (kNGlob - kQ0), st));
  HT_CHECK_CUDA(cudaMemset2DAsync(r->acc_img + kAyx, sizeof(double) * kNAcc, 0, sizeof(double) * 4, r->D.nimg, st));
  cudaError_t e = cudaErrorInvalidValue;
  const float2 *q0 = (const float2*)prby, *q1 = (const float2*)prbz;
  switch (r->D.n) {
#define X(S)                                                                                                      \
  case S:                                                                                                         \
    if (r->is_complex)                                                                                            \
      e = ndir == 2 ? hess_impl<S, float2, 2>(r, c, pos, mag, (const float2*)prb, data, cy, posy, q0, cz, posz, q1, st) \
                    : hess_impl<S, float2, 1>(r, c, pos, mag, (const float2*)prb, data, cy, posy, q0, cy, posy, q0, st); \
    else                                                                                                          \
      e = ndir == 2 ? hess_impl<S, float, 2>(r, c, pos, mag, (const float2*)prb, data, cy, posy, q0, cz, posz, q1, st)  \
                    : hess_impl<S, float, 1>(r, c, pos, mag, (const float2*)prb, data, cy, posy, q0, cy, posy, q0, st);  \
    break;
    HT_REC_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  const double qscale = 2.0 / r->ndata;
  k_casc_hess_combine<<<1, 256, 0, st>>>(r->acc_img, r->glob, posy, ndir == 2 ? posz : posy, ndir, r->D.nimg, qscale,
                                         accumulate, out);
  ::ht::count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}

// ====================================== objective without allocation
// For callers that cannot allocate device memory: their memory belongs to
// another allocator (a framework's caching pool, a serving loop with a fixed
// budget), or they must not call cudaMalloc/cudaFree because those calls can
// synchronise the whole device and stall other streams.  The scratch of this
// entry point is one file-scope device array of kNoAllocBytes, which every
// GPU that loads the library keeps until the process exits.
namespace ht {
constexpr size_t kNoAllocBytes = (size_t)32 << 20;  // 32 MiB
constexpr size_t kNoAllocAccBytes = 256;             // accumulators at the start
}  // namespace ht

static __device__ __align__(256) unsigned char g_noalloc_scratch[ht::kNoAllocBytes];

namespace ht {
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device; host code cannot use the array's name as a device address).
unsigned char* noalloc_scratch(int device) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (device < 0 || device >= kMaxDevices) return nullptr;
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      set_error(std::string("ht_rec_objective_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return nullptr;
    }
    g_noalloc_ptr[device] = static_cast<unsigned char*>(p);
  }
  return g_noalloc_ptr[device];
}
}  // namespace

template <int N, class T>
static cudaError_t noalloc_chunks(const ht_prop_s* prop, int nz, int nobj, int nzobj, int ndist, int ntheta,
                                  int per_chunk, const T* c, const float* pos, const float* mag, const float2* prb,
                                  const float* data, double* acc, float2* tmp, double* rows, double* imgs,
                                  cudaStream_t st) {
  const float2 *hw, *twn, *twz;
  prop_tables(prop, &hw, &twn, &twz);
  using CF = RowCfg<N>;
  const int smr = CF::SMEM + red_doubles<CF::T>(1, CF::THREADS) * (int)sizeof(double);
  cudaError_t e = N == kR512 ? cudaSuccess : allow_smem(k_casc_resid<N, 1>, smr);
  // chunks in angle order, each chunk's per-row sums reduced in a fixed order:
  // the objective is the same bit for bit on every call
  for (int th0 = 0; th0 < ntheta && e == cudaSuccess; th0 += per_chunk) {
    const int nt = std::min(per_chunk, ntheta - th0);
    const CascDims D{N, nz, nobj, nzobj, ndist, (long)nt * ndist};
    const long nrows = D.nimg * nz;
    e = launch_fwd<N, T>(D, c + (long)th0 * nzobj * nobj, pos + (long)th0 * ndist * 2, mag + (long)th0 * ndist, prb,
                         tmp, twn, st);
    if (e != cudaSuccess) break;
    if ((e = dct_cols(nz, false, tmp, D.nimg, N, hw, ndist, twz, st)) != cudaSuccess) break;
    const float* dch = data + (long)th0 * ndist * nz * N;
    if constexpr (N == kR512) {
      k_casc_resid512<1><<<(unsigned)((nrows + kR512Lines - 1) / kR512Lines), 32 * kR512Lines, 0, st>>>(
          tmp, nullptr, dch, nullptr, acc, rows, 0.f, D, twn);
    } else {
      k_casc_resid<N, 1><<<HT_ROWS_GRID(N, nrows), CF::THREADS, smr, st>>>(tmp, nullptr, dch, nullptr, acc, rows,
                                                                             0.f, D, twn);
    }
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    k_rows_img<<<(unsigned)D.nimg, kRedThreads, 0, st>>>(rows, 1, nz, imgs, nullptr, 0, 0, 0);
    count_launch();
    k_imgs_glob<<<1, kRedThreads, 0, st>>>(imgs, 1, D.nimg, acc, kF);
    count_launch();
    e = cudaGetLastError();
  }
  return e;
}
}  // namespace ht

extern "C" int ht_rec_objective_noalloc(ht_prop_s* prop, int nobj, int nzobj, int ntheta, int is_complex,
                                        const void* c, const float* pos, const float* mag, const void* prb,
                                        const float* data, double* fval, void* stream) {
  using namespace ht;
  HT_REQUIRE(prop && c && pos && mag && prb && data && fval, "ht_rec_objective_noalloc: null pointer");
  HT_REQUIRE(nobj > 0 && nzobj > 0 && ntheta > 0, "ht_rec_objective_noalloc: sizes must be positive");
  int n, nz, ndist;
  prop_dims(prop, &n, &nz, &ndist);
  bool n_ok = false;
#define X(S) n_ok = n_ok || (n == S);
  HT_REC_SIZES(X)
#undef X
  if (!n_ok) {
    set_error("ht_rec_objective_noalloc: n must be one of 32, 64, 128, 256, 384, 512, 768, 1024, 2048");
    return kUnsupported;
  }
  // per angle: its images (ndist*nz*n complex64), their per-row sums
  // (ndist*nz doubles) and per-image sums (ndist doubles)
  const size_t per_angle = sizeof(float2) * (size_t)ndist * nz * n + sizeof(double) * (size_t)ndist * (nz + 1);
  const size_t room = kNoAllocBytes - kNoAllocAccBytes;
  if (per_angle > room) {
    set_error("ht_rec_objective_noalloc: one angle needs " + std::to_string(per_angle) +
              " bytes of scratch (ndist*nz*n*8 + ndist*(nz+1)*8); the fixed scratch holds " + std::to_string(room) +
              " bytes (32 MiB minus 256)");
    return kBadArgument;
  }
  int device = 0;
  HT_CHECK_CUDA(cudaGetDevice(&device));
  unsigned char* base = noalloc_scratch(device);
  if (!base) return kCudaError;
  const int per_chunk = (int)std::min<size_t>(room / per_angle, (size_t)ntheta);
  double* acc = reinterpret_cast<double*>(base);
  float2* tmp = reinterpret_cast<float2*>(base + kNoAllocAccBytes);
  double* rows = reinterpret_cast<double*>(tmp + (size_t)per_chunk * ndist * nz * n);
  double* imgs = rows + (size_t)per_chunk * ndist * nz;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: clear the accumulators
  HT_CHECK_CUDA(cudaMemsetAsync(acc, 0, kNoAllocAccBytes, st));
  cudaError_t e = cudaErrorInvalidValue;
  switch (n) {
#define X(S)                                                                                                      \
  case S:                                                                                                         \
    e = is_complex ? noalloc_chunks<S, float2>(prop, nz, nobj, nzobj, ndist, ntheta, per_chunk, (const float2*)c, \
                                               pos, mag, (const float2*)prb, data, acc, tmp, rows, imgs, st)     \
                   : noalloc_chunks<S, float>(prop, nz, nobj, nzobj, ndist, ntheta, per_chunk, (const float*)c,   \
                                              pos, mag, (const float2*)prb, data, acc, tmp, rows, imgs, st);     \
    break;
    HT_REC_SIZES(X)
#undef X
    default:
      break;
  }
  HT_CHECK_CUDA(e);
  HT_CHECK_CUDA(cudaMemcpyAsync(fval, acc + kF, sizeof(double), cudaMemcpyDeviceToDevice, st));
  return kOk;
}
