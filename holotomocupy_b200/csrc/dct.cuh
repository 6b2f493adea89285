// Row-line DCT helpers shared by the propagator and the fused cascade.
//
// DCT-II (unnormalised, C[k] = sum_t f[t] cos(pi k (2t+1) / 2N)) by one
// N-point FFT (Makhoul): the input is reordered v[m] = f[2m],
// v[N-1-m] = f[2m+1]; after the FFT the outputs k and N-k are combined,
//   C[k] = 1/2 (w^k V[k] + w^-k V[N-k]),  C[N-k] = i/2 (w^k V[k] - w^-k V[N-k]),
// w = exp(-i pi / 2N).  DCT-III (the transpose, y[t] = sum_k G[k] cos(...))
// runs the transposed sequence: pre-combine, forward FFT, inverse reorder.
//
// All threads of a line must call these (they barrier over the line's
// threads, which are contiguous: line = threadIdx.x / T).
#pragma once
#include "lines.cuh"

namespace ht {

// Put input sample g of a DCT-II line (before dct2_finish).
template <int N>
__device__ __forceinline__ void dct2_put(const SmRow& sm, int g, float2 v) {
  sm.st(dct_perm_inv(g, N), v);
}

// FFT the staged line and write C[0..N) to dst (skipped when !valid).  The
// caller has synchronised after the last dct2_put.
template <int N, int T, class PL = Plan<N>>
__device__ __forceinline__ void dct2_finish(const SmRow& sm, int t, const float2* __restrict__ tw4, float2* dst,
                                            bool valid) {
  static_assert(T == PL::T, "T threads a line is the plan's");
  fft_line<N, false, PL>(sm, t, tw4, line_sync<T>());
  if (!valid) return;
  for (int k = t; k <= N / 2; k += T) {
    const float2 A = sm.ld(k), B = sm.ld(k == 0 ? 0 : N - k);
    const float2 w = __ldg(&tw4[k]);
    const float2 P = cmul(w, A), Q = cmulc(B, w);
    dst[k] = cscale(cadd(P, Q), 0.5f);
    if (k != 0 && k != N / 2) dst[N - k] = cscale(cmul_i(csub(P, Q)), 0.5f);
  }
}

// Load the DCT-III input G[0..N) from src, pre-combine and FFT.  Afterwards
// output sample g is sm.ld(dct_perm(g, N)).  Ends with a barrier over the
// line's threads.
template <int N, int T, class PL = Plan<N>>
__device__ __forceinline__ void dct3_start(const SmRow& sm, int t, const float2* __restrict__ tw4, const float2* src,
                                           bool valid) {
  static_assert(T == PL::T, "T threads a line is the plan's");
  // every load of the line is issued before the first store, so the thread
  // waits for global memory once
  constexpr int NM = (N / 2) / T + 1;  // m = t + i T covers 0..N/2
  float2 G[NM], H[NM];
#pragma unroll
  for (int i = 0; i < NM; ++i) {
    const int m = t + i * T;
    const bool ok = valid && m <= N / 2;
    G[i] = ok ? src[m] : make_float2(0.f, 0.f);
    H[i] = ok ? src[m == 0 ? 0 : N - m] : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int i = 0; i < NM; ++i) {
    const int m = t + i * T;
    if (m > N / 2) break;
    if (m == 0) {
      sm.st(0, G[i]);
    } else {
      const float2 w = __ldg(&tw4[m]);
      sm.st(m, cscale(cmul(w, cadd(G[i], cmul_i(H[i]))), 0.5f));
      if (m != N / 2) sm.st(N - m, cscale(cmulc(csub(G[i], cmul_i(H[i])), w), 0.5f));
    }
  }
  line_sync<T>()();
  fft_line<N, false, PL>(sm, t, tw4, line_sync<T>());
}

// Sums of K values over the T threads of each line, in double precision; the
// results are valid in thread t == 0 of the line.  red: shared scratch of
// K * blockDim.x doubles.  Every thread of the block must call it.
template <int T, int K>
__device__ __forceinline__ void line_sums(double (&v)[K], double* red, int line, int t) {
  if constexpr (T % 32 == 0) {
#pragma unroll
    for (int i = 0; i < K; ++i)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
    if constexpr (T > 32) {
      constexpr int W = T / 32;
      const int nl = blockDim.x / T;
      if ((t & 31) == 0)
#pragma unroll
        for (int i = 0; i < K; ++i) red[(i * nl + line) * W + t / 32] = v[i];
      __syncthreads();
      if (t == 0)
#pragma unroll
        for (int i = 0; i < K; ++i) {
          double s = 0.0;
          for (int w = 0; w < W; ++w) s += red[(i * nl + line) * W + w];
          v[i] = s;
        }
      __syncthreads();
    }
  } else {
#pragma unroll
    for (int i = 0; i < K; ++i) red[i * blockDim.x + threadIdx.x] = v[i];
    __syncthreads();
    if (t == 0)
#pragma unroll
      for (int i = 0; i < K; ++i) {
        double s = 0.0;
        for (int j = 0; j < T; ++j) s += red[i * blockDim.x + threadIdx.x + j];
        v[i] = s;
      }
    __syncthreads();
  }
}

}  // namespace ht
