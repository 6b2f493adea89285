// Fresnel propagator D / DT (reference: src/holotomocupy/propagation.py:70-112).
//
// The reference mirror-pads each [nz, n] image to [2nz, 2n], multiplies its
// 2-D FFT by fker[j] and crops the unnormalised inverse FFT.  The mirror pad
// is the half-sample-symmetric extension (circularly shifted by n/2, which
// commutes with the convolution), and fker is exactly even in kx and ky, so
// the same operator is
//
//     D(f) = T3_y T3_x ( Hw[j] * T2_y T2_x f ),   Hw = a_ky a_kx fker[j][ky, kx]
//
// with T2 the unnormalised DCT-II (sum f[t] cos(pi k (2t+1) / 2N)), T3 = T2^T,
// and a_0 = 2, a_k = 4 (k >= 1), over ky < nz, kx < n only.  DT uses conj(Hw).
// This touches [nz, n] instead of [2nz, 2n] samples, with the reference's own
// FP32 fker table, so results agree with the reference to FP32 rounding.
//
// Each DCT of length N is one N-point complex FFT (Makhoul): the input is
// reordered even/odd-reversed, transformed, and the outputs k and N-k are
// combined with exp(-i pi k / 2N) twiddles.  T3 is the transpose of that
// sequence (combine, FFT, reorder).
//
// Kernels: row DCT-II  ->  column [DCT-II, x Hw, DCT-III]  ->  row DCT-III.
// The column pass works in place, so D needs no scratch buffer.
#define HT_SCALAR_COMPLEX 1  // the column passes run faster on scalar complex adds (common.cuh)
#include "lines.cuh"
#include "row512.cuh"
#include "holotomo_b200_internal.h"

#include <vector>

namespace ht {

// ------------------------------------------------------------ row DCT-II
// in, out: [nrows, N]; out may alias in.
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_dct2_rows(const float2* in, float2* out, long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  constexpr int LS = SmRow::padded(N);
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < nrows;
  SmRow sm{smem + line * LS};
  const float2* src = in + row * N;
  for (int g = t; g < N; g += T) sm.st(dct_perm_inv(g, N), valid ? src[g] : make_float2(0.f, 0.f));
  __syncthreads();
  fft_line<N, false>(sm, t, tw4, line_sync<T>());
  if (!valid) return;
  float2* dst = out + row * N;
  for (int k = t; k <= N / 2; k += T) {
    const float2 A = sm.ld(k), B = sm.ld(k == 0 ? 0 : N - k);
    const float2 w = __ldg(&tw4[k]);
    const float2 P = cmul(w, A), Q = cmulc(B, w);
    dst[k] = cscale(cadd(P, Q), 0.5f);
    if (k != 0 && k != N / 2) dst[N - k] = cscale(cmul_i(csub(P, Q)), 0.5f);
  }
}

// ----------------------------------------------------------- row DCT-III
template <int N>
__global__ void __launch_bounds__(RowCfg<N>::THREADS)
k_dct3_rows(const float2* in, float2* out, long nrows, const float2* __restrict__ tw4) {
  constexpr int T = RowCfg<N>::T;
  constexpr int LS = SmRow::padded(N);
  extern __shared__ float2 smem[];
  const int line = threadIdx.x / T, t = threadIdx.x % T;
  const long row = (long)blockIdx.x * RowCfg<N>::LINES + line;
  const bool valid = row < nrows;
  SmRow sm{smem + line * LS};
  const float2* src = in + row * N;
  for (int m = t; m <= N / 2; m += T) {
    const float2 z = make_float2(0.f, 0.f);
    const float2 G = valid ? src[m] : z;
    const float2 H = valid ? src[m == 0 ? 0 : N - m] : z;
    if (m == 0) {
      sm.st(0, G);
    } else {
      const float2 w = __ldg(&tw4[m]);
      // V'[m] = 1/2 w^m (G[m] + i G[N-m]);  V'[N-m] = 1/2 conj(w^m) (G[m] - i G[N-m])
      sm.st(m, cscale(cmul(w, cadd(G, cmul_i(H))), 0.5f));
      if (m != N / 2) sm.st(N - m, cscale(cmulc(csub(G, cmul_i(H)), w), 0.5f));
    }
  }
  __syncthreads();
  fft_line<N, false>(sm, t, tw4, line_sync<T>());
  if (!valid) return;
  float2* dst = out + row * N;
  for (int g = t; g < N; g += T) dst[g] = sm.ld(dct_perm(g, N));
}

// ------------------------------------- column DCT-II, x table, DCT-III
// Column col of an image, read (ColIn) or written (ColOut) at position k of
// the reordered sequence, i.e. at image row dct_sample_at(k).
template <int NZ>
struct ColIn {
  const float2* p;  // row 0 of the column
  int n;
  bool valid;
  __device__ __forceinline__ float2 ld(int k) const {
    return valid ? p[(long)dct_sample_at(k, NZ) * n] : make_float2(0.f, 0.f);
  }
};
template <int NZ>
struct ColOut {
  float2* p;
  int n;
  bool valid;
  __device__ __forceinline__ void st(int k, float2 v) const {
    if (valid) p[(long)dct_sample_at(k, NZ) * n] = v;
  }
};

// data: [nimg, NZ, n] in place; H: [NZ, n] (the j-th distance's Hw).  The
// first FFT stage loads the block's C columns straight from global memory and
// the last one stores them there (a warp covers 32/C rows of C adjacent
// columns per access), so the column tile passes through shared memory only
// between stages.
// Two CTAs per SM up to 512 threads (ColCfg::MIN_BLOCKS; the register cap
// this sets, 64, spills a little at NZ = 2048): the block barriers of one CTA
// overlap the other's work (D at 2048^2 x 16 images 1.88 -> 1.67 ms, at
// 1024^2 x 32 0.80 -> 0.72 ms).
template <int NZ, bool CONJ>
__global__ void __launch_bounds__(ColCfg<NZ>::THREADS, ColCfg<NZ>::MIN_BLOCKS)
k_dct_cols(float2* data, int n, const float2* __restrict__ Hall, int ntab, const float2* __restrict__ tw4) {
  // image blockIdx.y uses table (blockIdx.y % ntab) of Hall [ntab, NZ, n]
  const float2* __restrict__ H = Hall + (long)(blockIdx.y % ntab) * NZ * n;
  constexpr int C = ColCfg<NZ>::C;
  constexpr int T = ColCfg<NZ>::T;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const bool valid = blockIdx.x * C + c < n;
  const int col = min((int)blockIdx.x * C + c, n - 1);
  float2* img = data + (long)blockIdx.y * NZ * n + col;
  SmCol<C> sm{tile + c};
  fft_line_from<NZ, false, typename ColCfg<NZ>::PL>(ColIn<NZ>{img, n, valid}, sm, t, tw4);
  for (int k = t; k <= NZ / 2; k += T) {
    const float2 A = sm.ld(k), B = sm.ld(k == 0 ? 0 : NZ - k);
    const float2 w = __ldg(&tw4[k]);
    const float2 P = cmul(w, A), Q = cmulc(B, w);
    float2 hk = __ldg(&H[(long)k * n + col]);
    if (CONJ) hk.y = -hk.y;
    const float2 Gk = cmul(cscale(cadd(P, Q), 0.5f), hk);
    if (k == 0) {
      sm.st(0, Gk);
    } else if (k == NZ / 2) {
      sm.st(k, cscale(cmul(w, cadd(Gk, cmul_i(Gk))), 0.5f));
    } else {
      float2 hn = __ldg(&H[(long)(NZ - k) * n + col]);
      if (CONJ) hn.y = -hn.y;
      const float2 Gn = cmul(cscale(cmul_i(csub(P, Q)), 0.5f), hn);
      sm.st(k, cscale(cmul(w, cadd(Gk, cmul_i(Gn))), 0.5f));
      sm.st(NZ - k, cscale(cmulc(csub(Gk, cmul_i(Gn)), w), 0.5f));
    }
  }
  __syncthreads();
  fft_line_to<NZ, false, typename ColCfg<NZ>::PL>(sm, ColOut<NZ>{img, n, valid}, t, tw4);
}

// ------------------- column pass at NZ = 512: the combine in registers
// One group of 32 threads per column, 16 samples a thread, radices 8, 8, 8.
// In the last stage of the DCT-II FFT and the first stage of the DCT-III FFT
// thread t owns the butterflies t and 64 - t (thread 0: 0 and 32), whose
// samples k = b + 64 j are closed under k -> 512 - k.  The k / N-k combine,
// the table product and the DCT-III pre-combine of both samples of a pair
// then happen in registers, so the spectrum makes no round trip through
// shared memory between the two transforms.
struct Col512 {
  static constexpr int N = 512, E = 16, T = 32, C = 8, THREADS = C * T;
  static constexpr int SMEM = N * C * (int)sizeof(float2);
};

// DCT-II output pair (X[k], X[N-k]) -> x Hw -> DCT-III input pair, 0 < k < N/2
// (the general case of the combine in k_dct_cols).
template <bool CONJ>
__device__ __forceinline__ void col_combine(float2& lo, float2& hi, int k, const float2* __restrict__ H, int n,
                                            const float2* __restrict__ tw4) {
  const float2 w = __ldg(&tw4[k]);
  const float2 P = cmul(w, lo), Q = cmulc(hi, w);
  float2 hk = __ldg(&H[(long)k * n]), hn = __ldg(&H[(long)(512 - k) * n]);
  if (CONJ) {
    hk.y = -hk.y;
    hn.y = -hn.y;
  }
  const float2 Gk = cmul(cscale(cadd(P, Q), 0.5f), hk);
  const float2 Gn = cmul(cscale(cmul_i(csub(P, Q)), 0.5f), hn);
  lo = cscale(cmul(w, cadd(Gk, cmul_i(Gn))), 0.5f);
  hi = cscale(cmulc(csub(Gk, cmul_i(Gn)), w), 0.5f);
}

template <bool CONJ>
__global__ void __launch_bounds__(Col512::THREADS)
k_dct_cols512(float2* data, int n, const float2* __restrict__ Hall, int ntab, const float2* __restrict__ tw4) {
  constexpr int N = 512, E = Col512::E, C = Col512::C;
  const float2* __restrict__ H0 = Hall + (long)(blockIdx.y % ntab) * N * n;
  extern __shared__ float2 tile[];
  const int c = threadIdx.x % C, t = threadIdx.x / C;
  const bool valid = blockIdx.x * C + c < n;
  const int col = min((int)blockIdx.x * C + c, n - 1);
  const float2* __restrict__ H = H0 + col;
  float2* img = data + (long)blockIdx.y * N * n + col;
  SmCol<C> sm{tile + c};
  const CtaSync sync{};
  float2 v[E];
  // DCT-II FFT: stages 1 (from global memory) and 2
  fft_stage<N, E, 8, 1, false, false, true>(v, SplitView<ColIn<N>, SmCol<C>>{ColIn<N>{img, n, valid}, sm}, t, tw4,
                                            sync);
  fft_stage<N, E, 8, 8, false, true, true>(v, sm, t, tw4, sync);
  // stage 3 (P = 64) for the butterflies b0, b1, kept in registers: v[8 s + j] = X[b_s + 64 j]
  const int b0 = t, b1 = (t == 0) ? 32 : 64 - t;
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int b = s ? b1 : b0;
#pragma unroll
    for (int j = 0; j < 8; ++j) v[8 * s + j] = sm.ld(b + 64 * j);
    float2 w[8];
    twiddles<8, false>(tw4, b, N, w);
#pragma unroll
    for (int j = 1; j < 8; ++j) v[8 * s + j] = cmul(v[8 * s + j], w[j]);
    Dft<8, false>::run(&v[8 * s]);
  }
  // combine, x Hw, pre-combine
  if (t != 0) {
    // pairs (b0 + 64 j, b1 + 64 (7 - j)); the first is the lower index for j < 4
#pragma unroll
    for (int j = 0; j < 4; ++j) col_combine<CONJ>(v[j], v[15 - j], t + 64 * j, H, n, tw4);
#pragma unroll
    for (int j = 4; j < 8; ++j) col_combine<CONJ>(v[15 - j], v[j], 64 - t + 64 * (7 - j), H, n, tw4);
  } else {
    // b0 = 0: 64 j pairs with 64 (8 - j); 0 and 256 pair with themselves
    {
      float2 h = __ldg(&H[0]);
      if (CONJ) h.y = -h.y;
      const float2 w = __ldg(&tw4[0]);
      v[0] = cmul(cscale(cadd(cmul(w, v[0]), cmulc(v[0], w)), 0.5f), h);
    }
    {
      float2 h = __ldg(&H[(long)256 * n]);
      if (CONJ) h.y = -h.y;
      const float2 w = __ldg(&tw4[256]);
      const float2 G = cmul(cscale(cadd(cmul(w, v[4]), cmulc(v[4], w)), 0.5f), h);
      v[4] = cscale(cmul(w, cadd(G, cmul_i(G))), 0.5f);
    }
#pragma unroll
    for (int j = 1; j < 4; ++j) col_combine<CONJ>(v[j], v[8 - j], 64 * j, H, n, tw4);
    // b1 = 32: 32 + 64 j pairs with 32 + 64 (7 - j)
#pragma unroll
    for (int j = 0; j < 4; ++j) col_combine<CONJ>(v[8 + j], v[15 - j], 32 + 64 * j, H, n, tw4);
  }
  sync();  // every stage-3 load is done before the stores below
  // DCT-III FFT: stage 1 (P = 1) on the same butterflies, then stages 2 and 3 (to global memory)
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int b = s ? b1 : b0;
    Dft<8, false>::run(&v[8 * s]);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm.st(b * 8 + j, v[8 * s + j]);
  }
  sync();
  fft_stage<N, E, 8, 8, false, true, true>(v, sm, t, tw4, sync);
  fft_stage<N, E, 8, 64, false, false, false>(v, SplitView<SmCol<C>, ColOut<N>>{sm, ColOut<N>{img, n, valid}}, t,
                                              tw4, sync);
}

// ---------------------------------------------------------------- launch
template <int N>
static cudaError_t launch_dct_rows(bool inverse, const float2* in, float2* out, long nrows,
                                   const float2* tw4, cudaStream_t st) {
  using CF = RowCfg<N>;
  const long grid = (nrows + CF::LINES - 1) / CF::LINES;
  if (inverse) {
    cudaError_t e = allow_smem(k_dct3_rows<N>, CF::SMEM);
    if (e != cudaSuccess) return e;
    k_dct3_rows<N><<<(unsigned)grid, CF::THREADS, CF::SMEM, st>>>(in, out, nrows, tw4); ::ht::count_launch();
  } else {
    cudaError_t e = allow_smem(k_dct2_rows<N>, CF::SMEM);
    if (e != cudaSuccess) return e;
    k_dct2_rows<N><<<(unsigned)grid, CF::THREADS, CF::SMEM, st>>>(in, out, nrows, tw4); ::ht::count_launch();
  }
  return cudaGetLastError();
}

template <int NZ>
static cudaError_t launch_dct_cols(bool conj, float2* data, long nimg, int n, const float2* H, int ntab,
                                   const float2* tw4, cudaStream_t st) {
  if constexpr (NZ == 512) {
    using CF = Col512;
    dim3 grid((n + CF::C - 1) / CF::C, (unsigned)nimg);
    auto kern = conj ? k_dct_cols512<true> : k_dct_cols512<false>;
    cudaError_t e = allow_smem(kern, CF::SMEM);
    if (e != cudaSuccess) return e;
    {
      KTimer kt("k_dct_cols", st, (double)nimg);
      kern<<<grid, CF::THREADS, CF::SMEM, st>>>(data, n, H, ntab, tw4);
    }
    ::ht::count_launch();
    return cudaGetLastError();
  }
  using CF = ColCfg<NZ>;
  dim3 grid((n + CF::C - 1) / CF::C, (unsigned)nimg);
  if (conj) {
    cudaError_t e = allow_smem(k_dct_cols<NZ, true>, CF::SMEM);
    if (e != cudaSuccess) return e;
    {
      KTimer kt("k_dct_cols", st, (double)nimg);
      k_dct_cols<NZ, true><<<grid, CF::THREADS, CF::SMEM, st>>>(data, n, H, ntab, tw4);
    }
    ::ht::count_launch();
  } else {
    cudaError_t e = allow_smem(k_dct_cols<NZ, false>, CF::SMEM);
    if (e != cudaSuccess) return e;
    {
      KTimer kt("k_dct_cols", st, (double)nimg);
      k_dct_cols<NZ, false><<<grid, CF::THREADS, CF::SMEM, st>>>(data, n, H, ntab, tw4);
    }
    ::ht::count_launch();
  }
  return cudaGetLastError();
}

cudaError_t dct_rows(int N, bool inverse, const float2* in, float2* out, long nrows, const float2* tw4,
                     cudaStream_t st) {
  switch (N) {
#define X(S) \
  case S:    \
    return launch_dct_rows<S>(inverse, in, out, nrows, tw4, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t dct_cols(int NZ, bool conj, float2* data, long nimg, int n, const float2* H, int ntab,
                     const float2* tw4, cudaStream_t st) {
  switch (NZ) {
#define X(S) \
  case S:    \
    return launch_dct_cols<S>(conj, data, nimg, n, H, ntab, tw4, st);
    HT_SIZE_CASES(X)
#undef X
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace ht

// ================================================================= C ABI
struct ht_prop_s {
  int n, nz, ndist, device;
  float2* hw;              // [ndist, nz, n] DCT-domain Fresnel tables
  const float2* tw_n;      // twiddles for the row length n
  const float2* tw_nz;     // twiddles for the column length nz
};

extern "C" int ht_prop_create(int n, int nz, int ndist, const void* fker_host, ht_prop_s** out) {
  using namespace ht;
  HT_REQUIRE(out != nullptr && fker_host != nullptr, "ht_prop_create: null pointer");
  HT_REQUIRE(n > 0 && nz > 0 && ndist > 0, "ht_prop_create: sizes must be positive");
  HT_REQUIRE(n % 2 == 0 && nz % 2 == 0, "ht_prop_create: n and nz must be even");
  if (!fft_size_supported(n) || !fft_size_supported(nz)) {
    set_error("ht_prop_create: n and nz must be one of 18,24,32,36,48,64,96,128,192,256,384,512,768,1024,1536,"
              "2048,3072,4096");
    return kUnsupported;
  }
  // Hw[j,ky,kx] = a_ky a_kx fker[j,ky,kx] for ky < nz, kx < n  (fker: [ndist, 2nz, 2n])
  const float2* fk = static_cast<const float2*>(fker_host);
  std::vector<float2> hw((size_t)ndist * nz * n);
  for (int j = 0; j < ndist; ++j)
    for (int ky = 0; ky < nz; ++ky)
      for (int kx = 0; kx < n; ++kx) {
        const float a = (ky == 0 ? 2.f : 4.f) * (kx == 0 ? 2.f : 4.f);
        const float2 f = fk[((size_t)j * 2 * nz + ky) * 2 * n + kx];
        hw[((size_t)j * nz + ky) * n + kx] = make_float2(a * f.x, a * f.y);
      }
  ht_prop_s* p = new ht_prop_s{n, nz, ndist, 0, nullptr, nullptr, nullptr};
  cudaGetDevice(&p->device);
  p->tw_n = twiddle_table(n, p->device);
  p->tw_nz = twiddle_table(nz, p->device);
  if (!p->tw_n || !p->tw_nz) {
    delete p;
    return kCudaError;
  }
  cudaError_t e = cudaMalloc(&p->hw, sizeof(float2) * hw.size());
  if (e == cudaSuccess) e = cudaMemcpy(p->hw, hw.data(), sizeof(float2) * hw.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    set_error(std::string("ht_prop_create: ") + cudaGetErrorString(e));
    if (p->hw) cudaFree(p->hw);
    delete p;
    return kCudaError;
  }
  *out = p;
  return kOk;
}

extern "C" int ht_prop_destroy(ht_prop_s* p) {
  if (!p) return ht::kOk;
  if (p->hw) cudaFree(p->hw);
  delete p;
  return ht::kOk;
}

namespace ht {
void prop_dims(const ht_prop_s* p, int* n, int* nz, int* ndist) {
  *n = p->n;
  *nz = p->nz;
  *ndist = p->ndist;
}

void prop_tables(const ht_prop_s* p, const float2** hw, const float2** twn, const float2** twz) {
  *hw = p->hw;
  *twn = p->tw_n;
  *twz = p->tw_nz;
}

int prop_apply(ht_prop_s* p, const void* in, void* out, long batch, int j, bool adjoint, cudaStream_t st) {
  HT_REQUIRE(p != nullptr, "propagator handle is null");
  HT_REQUIRE(in != nullptr && out != nullptr, "propagator: null data pointer");
  HT_REQUIRE(j >= 0 && j < p->ndist, "propagator: distance index out of range");
  HT_REQUIRE(batch >= 0, "propagator: negative batch");
  if (batch == 0) return kOk;
  const float2* src = static_cast<const float2*>(in);
  float2* dst = static_cast<float2*>(out);
  const float2* H = p->hw + (size_t)j * p->nz * p->n;
  HT_CHECK_CUDA(dct_rows(p->n, false, src, dst, batch * p->nz, p->tw_n, st));
  HT_CHECK_CUDA(dct_cols(p->nz, adjoint, dst, batch, p->n, H, 1, p->tw_nz, st));
  HT_CHECK_CUDA(dct_rows(p->n, true, dst, dst, batch * p->nz, p->tw_n, st));
  return kOk;
}
}  // namespace ht

extern "C" int ht_prop_D(ht_prop_s* p, const void* in, void* out, long batch, int j, void* stream) {
  return ht::prop_apply(p, in, out, batch, j, false, static_cast<cudaStream_t>(stream));
}

extern "C" int ht_prop_DT(ht_prop_s* p, const void* in, void* out, long batch, int j, void* stream) {
  return ht::prop_apply(p, in, out, batch, j, true, static_cast<cudaStream_t>(stream));
}
