// Launch helpers shared by the operators: block-shape choices for row and
// column line transforms, the size dispatch, and dynamic shared memory set-up.
#pragma once
#include "fft.cuh"

namespace ht {

// Rows per CTA for a row pass of length N: about 256 threads per CTA.
template <int N>
struct RowCfg {
  static constexpr int T = Plan<N>::T;
  static constexpr int LINES = (T >= 256) ? 1 : (256 / T);
  static constexpr int THREADS = LINES * T;
  static constexpr int SMEM = LINES * SmRow::padded(N) * (int)sizeof(float2);
  // lines of whole warps synchronise on named barriers 1..15 (LineSync)
  static_assert(T % 32 != 0 || LINES <= 15, "at most 15 line barriers per block");
};

// Columns per CTA for a column pass of length N (tile N x C in shared memory;
// at N >= 2048 the 4-column tile's rows are swizzled, see SmCol).
template <int N>
struct ColCfg {
  using PL = ColPlan<N>;
  static constexpr int T = PL::T;
  static constexpr int C = (N >= 2048) ? 4 : ((N >= 256) ? 8 : 16);
  static constexpr int THREADS = C * T;
  static constexpr int SMEM = N * C * (int)sizeof(float2);
  // two CTAs per SM where that leaves 64 registers a thread (one CTA's block
  // barriers then overlap the other's work); the 1024-thread tiles keep one
  static constexpr int MIN_BLOCKS = THREADS <= 512 ? 2 : 1;
};

// Raise the dynamic shared-memory limit of a kernel (no-op below 48 KB).  The
// attribute is set once per (device, kernel, size), so the launches that
// follow (including ones recorded into CUDA graphs) make no further runtime
// calls.
bool smem_attr_done(const void* kernel, int bytes);
void smem_attr_mark(const void* kernel, int bytes);
template <class K>
inline cudaError_t allow_smem(K kernel, int bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  const void* key = reinterpret_cast<const void*>(kernel);
  if (smem_attr_done(key, bytes)) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) smem_attr_mark(key, bytes);
  return e;
}

// A column of a [rows, ncols] image in global memory, as a line view for the
// first (GColIn) or last (GColOut) stage of a column transform; an invalid
// column (past the image's edge) reads zeros and stores nothing.
struct GColIn {
  const float2* p;  // row 0 of the column
  int ncols;
  bool valid;
  __device__ __forceinline__ float2 ld(int k) const { return valid ? p[(long)k * ncols] : make_float2(0.f, 0.f); }
};
struct GColOut {
  float2* p;
  int ncols;
  bool valid;
  __device__ __forceinline__ void st(int k, float2 v) const {
    if (valid) p[(long)k * ncols] = v;
  }
};

// Position of input sample g after the even/odd-reversed reordering used by
// the DCT-II (v[m] = f[2m], v[N-1-m] = f[2m+1]).
__device__ __forceinline__ int dct_perm_inv(int g, int N) { return (g & 1) ? (N - 1 - (g >> 1)) : (g >> 1); }
// Sample of the reordered sequence that lands on output position g.
__device__ __forceinline__ int dct_perm(int g, int N) { return dct_perm_inv(g, N); }
// Inverse of dct_perm_inv: the input sample at position p of the reordered
// sequence (and the output sample that position p lands on).
__device__ __forceinline__ int dct_sample_at(int p, int N) { return (2 * p < N) ? 2 * p : 2 * (N - 1 - p) + 1; }

}  // namespace ht

// Runtime size -> template dispatch over the supported transform lengths.
#define HT_SIZE_CASES(X) \
  X(18) X(24) X(32) X(36) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) \
  X(768) X(1024) X(1536) X(2048) X(3072) X(4096)
