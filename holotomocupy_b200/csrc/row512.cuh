// Row DCTs of length 512 by one warp per line: 16 samples a thread, radices
// 8-8-8 (stage P = 1, 8, 64), the line in a padded shared-memory row.
//
// Position p of the FFT sequence is held, after the last stage of an FFT and
// before the first, by thread p % 32 at register 8 ((p / 32) % 2) + p / 64:
// the butterflies b = t + 32 s of the first and last stages own the samples
// b + 64 j.  A pixel's DCT-III output and its DCT-II input sit at the same
// position (image sample dct_sample_at(p)), so a row kernel can take the
// pixels from one transform's last stage and give them to the next
// transform's first stage in registers.
//
// The DCT's k / N-k combines need both samples of a pair: for them thread t
// owns the butterflies t and 64 - t (thread 0: 0 and 32), whose samples are
// closed under p -> 512 - p.  The DCT-III input combine is done so before its
// first stage, and the DCT-II output combine after its last stage, straight
// from / to global memory.
#pragma once
#include "fft.cuh"
#include "lines.cuh"

namespace ht {

struct WarpSync {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
// A store view that drops its values (a last stage whose outputs stay in
// registers).
struct NullView {
  __device__ __forceinline__ void st(int, float2) const {}
};

constexpr int kR512 = 512;
__device__ __forceinline__ int r512_b1(int t) { return t == 0 ? 32 : 64 - t; }

// Position of register i of thread t after a last stage / before a first stage
// with the plain mapping.
__device__ __forceinline__ int r512_pos(int t, int i) { return t + 32 * (i / 8) + 64 * (i % 8); }

// DCT-III input of one line: G (the spectrum row, global) combined into the
// FFT input V'[m] = w^m (G[m] + i G[N-m]) / 2, V'[N-m] = conj(w^m) (G[m] - i
// G[N-m]) / 2 (V'[0] = G[0]), then the first FFT stage, stored to sm.  Ends
// with a warp barrier.
__device__ __forceinline__ void r512_dct3_head(float2 (&v)[16], const float2* __restrict__ G, bool valid,
                                               const SmRow& sm, int t, const float2* __restrict__ tw4) {
  const int b0 = t, b1 = r512_b1(t);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    v[j] = valid ? G[b0 + 64 * j] : make_float2(0.f, 0.f);
    v[8 + j] = valid ? G[b1 + 64 * j] : make_float2(0.f, 0.f);
  }
  auto pre = [&](float2& lo, float2& hi, int m) {
    const float2 w = __ldg(&tw4[m]);
    const float2 a = cscale(cmul(w, cadd(lo, cmul_i(hi))), 0.5f);
    hi = cscale(cmulc(csub(lo, cmul_i(hi)), w), 0.5f);
    lo = a;
  };
  if (t != 0) {
    // pairs (b0 + 64 j, b1 + 64 (7 - j)); the first is below N/2 for j < 4
#pragma unroll
    for (int j = 0; j < 4; ++j) pre(v[j], v[15 - j], t + 64 * j);
#pragma unroll
    for (int j = 4; j < 8; ++j) pre(v[15 - j], v[j], 64 - t + 64 * (7 - j));
  } else {
    // b0 = 0: 64 j pairs with 64 (8 - j); 0 and 256 with themselves
    const float2 w = __ldg(&tw4[256]);
    v[4] = cscale(cmul(w, cadd(v[4], cmul_i(v[4]))), 0.5f);
#pragma unroll
    for (int j = 1; j < 4; ++j) pre(v[j], v[8 - j], 64 * j);
    // b1 = 32: 32 + 64 j pairs with 32 + 64 (7 - j)
#pragma unroll
    for (int j = 0; j < 4; ++j) pre(v[8 + j], v[15 - j], 32 + 64 * j);
  }
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int b = s ? b1 : b0;
    Dft<8, false>::run(&v[8 * s]);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm.st(b * 8 + j, v[8 * s + j]);
  }
  __syncwarp();
}

// Stages 2 and 3 of a line whose stage 1 is in sm; the result stays in
// registers (plain mapping: v[i] is position r512_pos(t, i)).
__device__ __forceinline__ void r512_finish_to_regs(float2 (&v)[16], const SmRow& sm, int t,
                                                    const float2* __restrict__ tw4) {
  const WarpSync ws{};
  fft_stage<kR512, 16, 8, 8, false, true, true>(v, sm, t, tw4, ws);
  fft_stage<kR512, 16, 8, 64, false, false, false>(v, SplitView<SmRow, NullView>{sm, NullView{}}, t, tw4, ws);
}

// DCT-II of the line whose FFT input is in registers (plain mapping), written
// to dst (when valid): stages 1 and 2 through sm, stage 3 on the butterflies
// t and 64 - t, the output combine dst[k] = (P + Q) / 2, dst[N-k] = i (P - Q) / 2
// (P = w^k X[k], Q = conj(w^k) X[N-k]) in registers.  sm may still be read by
// the line's previous stage: the first thing done is a warp barrier.
__device__ __forceinline__ void r512_dct2_tail(float2 (&v)[16], const SmRow& sm, int t,
                                               const float2* __restrict__ tw4, float2* __restrict__ dst, bool valid) {
  __syncwarp();
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int b = t + 32 * s;
    Dft<8, false>::run(&v[8 * s]);
#pragma unroll
    for (int j = 0; j < 8; ++j) sm.st(b * 8 + j, v[8 * s + j]);
  }
  __syncwarp();
  fft_stage<kR512, 16, 8, 8, false, true, true>(v, sm, t, tw4, WarpSync{});
  const int b0 = t, b1 = r512_b1(t);
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const int b = s ? b1 : b0;
#pragma unroll
    for (int j = 0; j < 8; ++j) v[8 * s + j] = sm.ld(b + 64 * j);
    float2 w[8];
    twiddles<8, false>(tw4, b, kR512, w);
#pragma unroll
    for (int j = 1; j < 8; ++j) v[8 * s + j] = cmul(v[8 * s + j], w[j]);
    Dft<8, false>::run(&v[8 * s]);
  }
  if (!valid) return;
  auto put = [&](const float2 A, const float2 B, int k) {
    const float2 w = __ldg(&tw4[k]);
    const float2 P = cmul(w, A), Q = cmulc(B, w);
    dst[k] = cscale(cadd(P, Q), 0.5f);
    if (k != 0 && k != kR512 / 2) dst[kR512 - k] = cscale(cmul_i(csub(P, Q)), 0.5f);
  };
  if (t != 0) {
#pragma unroll
    for (int j = 0; j < 4; ++j) put(v[j], v[15 - j], t + 64 * j);
#pragma unroll
    for (int j = 4; j < 8; ++j) put(v[15 - j], v[j], 64 - t + 64 * (7 - j));
  } else {
    put(v[0], v[0], 0);
    put(v[4], v[4], 256);
#pragma unroll
    for (int j = 1; j < 4; ++j) put(v[j], v[8 - j], 64 * j);
#pragma unroll
    for (int j = 0; j < 4; ++j) put(v[8 + j], v[15 - j], 32 + 64 * j);
  }
}

// Sum of a double over the warp (lane 0 has it).
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  return x;
}

}  // namespace ht
