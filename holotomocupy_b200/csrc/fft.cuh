// Shared-memory Stockham FFT for one line of N complex samples held by a
// group of T = N/E threads (E samples per thread in registers).
//
// Every stage of radix R reads R samples per butterfly from shared memory at
// stride N/R (coalesced across the group), multiplies by the twiddles
// W_{P R}^{i j}, runs an R-point DFT in registers and writes the results to
// their self-sorting positions (b - i) R + i + j P, where P is the product of
// the radices already applied and i = b mod P.  The result is in natural
// order, so no bit reversal pass is needed.
//
// The line lives in shared memory behind an accessor (row lines are
// contiguous with one pad slot every 16 samples; column lines of a tile are
// strided by the tile width), so the same code serves row and column passes.
#pragma once
#include "common.cuh"

#include <type_traits>

namespace ht {

// ------------------------------------------------------- small DFT kernels
template <int R, bool INV>
struct Dft;

template <bool INV>
struct Dft<2, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Dft<3, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    const float s3 = 0.86602540378443864676f;  // sqrt(3)/2
    float2 a = v[0], b = v[1], c = v[2];
    float2 t1 = cadd(b, c), t2 = csub(b, c);
    float2 m1 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
    float2 m2 = rot<INV>(cscale(t2, s3));
    v[0] = cadd(a, t1);
    v[1] = cadd(m1, m2);
    v[2] = csub(m1, m2);
  }
};

template <bool INV>
struct Dft<4, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    float2 t2 = cadd(v[1], v[3]), t3 = rot<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV>
struct Dft<8, INV> {
  static __device__ __forceinline__ void run(float2* v) {
    const float r = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV>::run(e);
    Dft<4, INV>::run(o);
    // W8^1 = (1 -/+ i)/sqrt2, W8^2 = -/+ i, W8^3 = (-1 -/+ i)/sqrt2
    float2 o1 = INV ? make_float2(r * (o[1].x - o[1].y), r * (o[1].x + o[1].y))
                    : make_float2(r * (o[1].x + o[1].y), r * (o[1].y - o[1].x));
    float2 o2 = rot<INV>(o[2]);
    float2 o3 = INV ? make_float2(-r * (o[3].x + o[3].y), r * (o[3].x - o[3].y))
                    : make_float2(r * (o[3].y - o[3].x), -r * (o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

// ----------------------------------------------------- shared-memory views
// Row line: contiguous, one pad slot every 16 samples (bank-conflict free for
// the stride-R writes of the first stages).
struct SmRow {
  float2* p;
  static __host__ __device__ constexpr int padded(int n) { return n + (n >> 4); }
  __device__ __forceinline__ float2 ld(int k) const { return p[k + (k >> 4)]; }
  __device__ __forceinline__ void st(int k, float2 v) const { p[k + (k >> 4)] = v; }
  // sample k + 16 m sits 17 m slots after sample k: a stage whose strides are
  // multiples of 16 forms one padded index per butterfly and adds constants
  __device__ __forceinline__ float2 ld_pad(int pk) const { return p[pk]; }
  __device__ __forceinline__ void st_pad(int pk, float2 v) const { p[pk] = v; }
};

// Column line inside a [N][C] tile (row-major, C columns side by side).  For
// C = 4 (32-byte rows) row k is stored at k ^ ((k >> 3) & 3): the rows 8
// apart that the first radix-8 stage writes together then fall on different
// banks, and consecutive rows stay on different banks.
template <int C>
__host__ __device__ __forceinline__ int col_row(int k) {
  return (C == 4) ? (k ^ ((k >> 3) & 3)) : k;
}
template <int C>
struct SmCol {
  float2* p;  // points at column c of row 0
  __device__ __forceinline__ float2 ld(int k) const { return p[col_row<C>(k) * C]; }
  __device__ __forceinline__ void st(int k, float2 v) const { p[col_row<C>(k) * C] = v; }
};

// --------------------------------------------------------------- the plan
template <int... Rs>
struct Radices {};

// A line plan: samples per thread E (so N / E threads a line) and the radix
// sequence (product = N, every radix divides E).
template <int NN, int EE, int... Rs>
struct PlanOf {
  static constexpr int E = EE;
  static constexpr int T = NN / EE;
  using R = Radices<Rs...>;
};
// Plan<N>: the plan of every row line of N samples.
template <int N>
struct Plan;
#define HT_PLAN(NN, EE, ...) \
  template <>                \
  struct Plan<NN> : PlanOf<NN, EE, __VA_ARGS__> {};
HT_PLAN(18, 6, 2, 3, 3)
HT_PLAN(24, 12, 4, 3, 2)
HT_PLAN(32, 8, 8, 4)
HT_PLAN(36, 12, 4, 3, 3)
HT_PLAN(48, 12, 4, 4, 3)
HT_PLAN(64, 8, 8, 8)
HT_PLAN(96, 24, 8, 4, 3)
HT_PLAN(128, 8, 8, 4, 4)
HT_PLAN(192, 24, 8, 8, 3)
HT_PLAN(256, 8, 8, 8, 4)
HT_PLAN(384, 12, 4, 4, 4, 3, 2)   // 12 samples a thread: the stencil row kernels keep their occupancy
HT_PLAN(512, 8, 8, 8, 8)
HT_PLAN(768, 12, 4, 4, 4, 4, 3)
HT_PLAN(1024, 16, 8, 8, 8, 2)
HT_PLAN(1536, 24, 8, 8, 8, 3)
HT_PLAN(2048, 16, 8, 8, 8, 4)
HT_PLAN(3072, 24, 8, 8, 8, 2, 3)
HT_PLAN(4096, 16, 8, 8, 8, 8)
#undef HT_PLAN

// ColPlan<N>: the plan of the column passes (a tile of columns per CTA, no
// stencil work beside the transform): the row plan, except at 384 samples,
// where the 24-sample plan's four stages beat the 12-sample plan's five
// (column pass at 384 x 384 x 2688 images: 14.3 ms against 15.5 ms).
template <int N>
struct ColPlan : Plan<N> {};
template <>
struct ColPlan<384> : PlanOf<384, 24, 8, 8, 3, 2> {};
template <>
struct ColPlan<768> : PlanOf<768, 24, 8, 8, 4, 3> {};

// StPlan<N>: the plan of the stencil row kernels of the fused cascade, whose
// rows carry the stencil work beside the transform (so more threads a line
// pay): the row plan, except at 1024 samples, where 8 samples a thread (128
// threads a line) beat 16 (BH iteration at 1024^2 x 256 x 4: 273 against
// 283 ms); the other 1024-sample lines (the Radon transform's at n = 512)
// keep 16, which is faster for them.
template <int N>
struct StPlan : Plan<N> {};
template <>
struct StPlan<1024> : PlanOf<1024, 8, 8, 8, 8, 2> {};

// ------------------------------------------------------ synchronisation
// Barrier between the stages of one line's transform.  CtaSync: the whole
// block (lines whose data other lines read).  LineSync<T>: only the T
// threads of the line, which are contiguous (line = threadIdx.x / T): the
// warp when T divides 32 (the line lies inside one warp), a named barrier
// when T is a multiple of 32, else (T = 3: lines straddle warps) the block.
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
template <int T>
struct LineSync {
  int id;  // line index within the block (named barrier id + 1)
  __device__ __forceinline__ void operator()() const {
    if constexpr (32 % T == 0) {
      const unsigned lanes = min(32u, blockDim.x - (threadIdx.x & ~31u));
      __syncwarp(lanes == 32u ? 0xffffffffu : ((1u << lanes) - 1u));
    } else if constexpr (T % 32 == 0) {
      asm volatile("bar.sync %0, %1;" ::"r"(id + 1), "n"(T) : "memory");
    } else {
      __syncthreads();
    }
  }
};
template <int T>
__device__ __forceinline__ LineSync<T> line_sync() {
  return LineSync<T>{(int)(threadIdx.x / T)};
}

// Twiddles W^(a j), j = 1..R-1, from two table reads: W^a and W^(2a) are
// read, the others are products of them (a few ulps from the table values).
template <int R, bool INV>
__device__ __forceinline__ void twiddles(const float2* __restrict__ tw4, int a, int N, float2 (&w)[R]) {
  w[0] = make_float2(1.f, 0.f);
  float2 w1 = __ldg(&tw4[4 * a]);
  if (INV) w1.y = -w1.y;
  w[1] = w1;
  if constexpr (R > 2) {
    float2 w2 = __ldg(&tw4[4 * ((2 * a) % N)]);
    if (INV) w2.y = -w2.y;
    w[2] = w2;
    if constexpr (R > 3) {
      w[3] = cmul(w1, w2);
      if constexpr (R > 4) {
        const float2 w4 = cmul(w2, w2);
        w[4] = w4;
        w[5] = cmul(w1, w4);
        w[6] = cmul(w2, w4);
        w[7] = cmul(w[3], w4);
      }
    }
  }
}

// Loads through one view, stores through another: a first stage that reads
// its line from global memory, or a last stage that writes it there.
template <class L, class S>
struct SplitView {
  L l;
  S s;
  __device__ __forceinline__ float2 ld(int k) const { return l.ld(k); }
  __device__ __forceinline__ void st(int k, float2 v) const { s.st(k, v); }
};

// ------------------------------------------------------------- one stage
// tw4: table of exp(-2 pi i m / (4N)); W_N^a = tw4[4a].  SYNC_MID: barrier
// between the loads and the stores (needed when both are the same shared
// line); SYNC_END: barrier after the stores (needed when the next stage
// reads them).
template <int N, int E, int R, int P, bool INV, bool SYNC_MID, bool SYNC_END, class SM, class SY>
__device__ __forceinline__ void fft_stage(float2 (&v)[E], const SM& sm, int t,
                                          const float2* __restrict__ tw4, const SY& sync) {
  constexpr int T = N / E;
  constexpr int NB = E / R;
  constexpr int NR = N / R;
  static_assert(E % R == 0, "radix must divide the samples per thread");
  static_assert(R <= 8, "twiddles() covers radices up to 8");
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    const int b = t + s * T;
    if constexpr (std::is_same<SM, SmRow>::value && NR % 16 == 0) {
      const int pb = b + (b >> 4);
#pragma unroll
      for (int j = 0; j < R; ++j) v[s * R + j] = sm.ld_pad(pb + j * (NR + NR / 16));
    } else {
#pragma unroll
      for (int j = 0; j < R; ++j) v[s * R + j] = sm.ld(b + j * NR);
    }
  }
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    const int b = t + s * T;
    if constexpr (P > 1) {
      const int i = b % P;
      float2 w[R];
      twiddles<R, INV>(tw4, i * (N / (P * R)), N, w);
#pragma unroll
      for (int j = 1; j < R; ++j) v[s * R + j] = cmul(v[s * R + j], w[j]);
    }
    Dft<R, INV>::run(&v[s * R]);
  }
  if constexpr (SYNC_MID) sync();
#pragma unroll
  for (int s = 0; s < NB; ++s) {
    const int b = t + s * T;
    const int i = (P > 1) ? (b % P) : 0;
    if constexpr (std::is_same<SM, SmRow>::value && P % 16 == 0) {
      const int k0 = (b - i) * R + i;
      const int pk = k0 + (k0 >> 4);
#pragma unroll
      for (int j = 0; j < R; ++j) sm.st_pad(pk + j * (P + P / 16), v[s * R + j]);
    } else {
#pragma unroll
      for (int j = 0; j < R; ++j) sm.st((b - i) * R + i + j * P, v[s * R + j]);
    }
  }
  if constexpr (SYNC_END) sync();
}

template <int N, int E, int P, bool INV, class SM, class SY, int R, int... Rs>
__device__ __forceinline__ void fft_stages(float2 (&v)[E], const SM& sm, int t,
                                           const float2* __restrict__ tw4, const SY& sync, Radices<R, Rs...>) {
  constexpr bool LAST = sizeof...(Rs) == 0;
  fft_stage<N, E, R, P, INV, true, true>(v, sm, t, tw4, sync);
  if constexpr (!LAST) fft_stages<N, E, P * R, INV>(v, sm, t, tw4, sync, Radices<Rs...>{});
}

// As fft_stages, with the first stage loading from `in` (GIN) and/or the last
// stage storing to `out` (GOUT) instead of the shared line: a stage that
// reads global memory needs no barrier before its stores, and a stage that
// writes global memory none at all.
template <int N, int E, int P, bool INV, bool GIN, bool GOUT, class IN, class SM, class OUT, class SY, int R,
          int... Rs>
__device__ __forceinline__ void fft_stages_io(float2 (&v)[E], const IN& in, const SM& sm, const OUT& out, int t,
                                              const float2* __restrict__ tw4, const SY& sync, Radices<R, Rs...>) {
  constexpr bool FIRST = P == 1;
  constexpr bool LAST = sizeof...(Rs) == 0;
  static_assert(!(FIRST && LAST), "a line transform here has at least two stages");
  if constexpr (FIRST && GIN) {
    fft_stage<N, E, R, P, INV, false, true>(v, SplitView<IN, SM>{in, sm}, t, tw4, sync);
  } else if constexpr (LAST && GOUT) {
    fft_stage<N, E, R, P, INV, false, false>(v, SplitView<SM, OUT>{sm, out}, t, tw4, sync);
  } else {
    fft_stage<N, E, R, P, INV, true, true>(v, sm, t, tw4, sync);
  }
  if constexpr (!LAST) fft_stages_io<N, E, P * R, INV, GIN, GOUT>(v, in, sm, out, t, tw4, sync, Radices<Rs...>{});
}

// In-place FFT of the line held in shared memory (natural order in, natural
// order out).  All T threads of the line must call it, and every thread the
// barrier `sync` covers (it barriers between stages).  The caller
// synchronises before (so the input is complete); the result is complete
// for the threads `sync` covers on return.
template <int N, bool INV, class PL = Plan<N>, class SM, class SY = CtaSync>
__device__ __forceinline__ void fft_line(const SM& sm, int t, const float2* __restrict__ tw4,
                                         const SY& sync = SY{}) {
  float2 v[PL::E];
  fft_stages<N, PL::E, 1, INV>(v, sm, t, tw4, sync, typename PL::R{});
}

// FFT of a line read from `in` (any view with ld(k): sample k of the line),
// result left in shared memory (complete for the threads `sync` covers).  No
// barrier is needed before it.
template <int N, bool INV, class PL = Plan<N>, class IN, class SM, class SY = CtaSync>
__device__ __forceinline__ void fft_line_from(const IN& in, const SM& sm, int t, const float2* __restrict__ tw4,
                                              const SY& sync = SY{}) {
  float2 v[PL::E];
  fft_stages_io<N, PL::E, 1, INV, true, false>(v, in, sm, sm, t, tw4, sync, typename PL::R{});
}

// FFT of a line read from `in` and written to `out` (the first stage loads
// from `in`, the last stage stores to `out`, the stages between pass through
// shared memory); no barrier is needed before it, none is made after it.
template <int N, bool INV, class PL = Plan<N>, class IN, class SM, class OUT, class SY = CtaSync>
__device__ __forceinline__ void fft_line_io(const IN& in, const SM& sm, const OUT& out, int t,
                                            const float2* __restrict__ tw4, const SY& sync = SY{}) {
  float2 v[PL::E];
  fft_stages_io<N, PL::E, 1, INV, true, true>(v, in, sm, out, t, tw4, sync, typename PL::R{});
}

// FFT of a line in shared memory (the caller synchronised after writing it),
// result stored through `out` (any view with st(k, v)); the line is not
// barriered afterwards.
template <int N, bool INV, class PL = Plan<N>, class SM, class OUT, class SY = CtaSync>
__device__ __forceinline__ void fft_line_to(const SM& sm, const OUT& out, int t, const float2* __restrict__ tw4,
                                            const SY& sync = SY{}) {
  float2 v[PL::E];
  fft_stages_io<N, PL::E, 1, INV, false, true>(v, sm, sm, out, t, tw4, sync, typename PL::R{});
}

}  // namespace ht
