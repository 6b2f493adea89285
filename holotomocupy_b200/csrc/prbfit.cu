// Probe-fit regulariser lam |||D prb| - ref||^2 / (ndist nz n) on the device
// (reference: Rec.gradient_prbfit and Rec.hessian_prbfit,
// src/holotomocupy/rec_mpi.py:365-398): its gradient and its Hessian forms
// with the propagator kernels and FP64 reductions, no host round trip, so a
// BH iteration with the term can be recorded into a CUDA graph.
#include <algorithm>

#include "common.cuh"
#include "holotomo_b200_internal.h"

namespace ht {
namespace {

constexpr int kPfThreads = 256;

unsigned pf_grid(long n) {
  const long g = (n + kPfThreads - 1) / kPfThreads;
  return (unsigned)std::min<long>(std::max<long>(g, 1), 148L * 8);
}

// t = 2 (t - ref t / |t|)  (rec_mpi.py:372-374: 2 * (tmp - ref * tmp / |tmp|))
__global__ void __launch_bounds__(kPfThreads) k_prbfit_resid(float2* __restrict__ t, const float* __restrict__ ref,
                                                             long n) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float2 v = t[i];
    const float a = sqrtf(v.x * v.x + v.y * v.y);
    const float r = ref[i];
    t[i] = make_float2(2.f * (v.x - r * (v.x / a)), 2.f * (v.y - r * (v.y / a)));
  }
}

// Per-block FP64 partial sums part[block][0..2] of the forms of the pairs
// (a, a), (a, b), (b, b): sum (1 - d0) Re(u conj w) + d0 Re(conj(l) u) Re(conj(l) w),
// l = p / |p|, d0 = ref / |p| (rec_mpi.py:390-396); b == nullptr: (a, a) only.
__global__ void __launch_bounds__(kPfThreads) k_prbfit_forms(const float2* __restrict__ p, const float2* __restrict__ a,
                                                             const float2* __restrict__ b, const float* __restrict__ ref,
                                                             long n, double* __restrict__ part) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float2 pv = p[i], u = a[i];
    const float m = sqrtf(pv.x * pv.x + pv.y * pv.y);
    const float2 l = make_float2(pv.x / m, pv.y / m);
    const float d0 = ref[i] / m;
    const float lu = l.x * u.x + l.y * u.y;
    s0 += (double)((1.f - d0) * (u.x * u.x + u.y * u.y) + d0 * lu * lu);
    if (b) {
      const float2 w = b[i];
      const float lw = l.x * w.x + l.y * w.y;
      s1 += (double)((1.f - d0) * (u.x * w.x + u.y * w.y) + d0 * lu * lw);
      s2 += (double)((1.f - d0) * (w.x * w.x + w.y * w.y) + d0 * lw * lw);
    }
  }
  __shared__ double red[3][kPfThreads / 32];
  double v[3] = {s0, s1, s2};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    if ((threadIdx.x & 31) == 0) red[k][threadIdx.x / 32] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int w = 0; w < kPfThreads / 32; ++w) t += red[threadIdx.x][w];
    part[blockIdx.x * 3 + threadIdx.x] = t;
  }
}

// The partials summed in block order, times 2 scale; slots = 0: out[0..2] =
// the three forms; slots = 1: added to the BH Hessian slots {H(g,g),
// H_ref(g,e), H(e,e), H_sym(g,e)} (the term is symmetric: both H(g,e) slots
// get the (a, b) form).
__global__ void k_prbfit_finish(const double* __restrict__ part, int nblk, double scale, int slots,
                                double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double f[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < nblk; ++i)
    for (int k = 0; k < 3; ++k) f[k] += part[i * 3 + k];
  for (int k = 0; k < 3; ++k) f[k] *= 2.0 * scale;
  if (slots) {
    out[0] += f[0];
    out[1] += f[1];
    out[2] += f[2];
    out[3] += f[1];
  } else {
    out[0] = f[0];
    out[1] = f[1];
    out[2] = f[2];
  }
}

}  // namespace
}  // namespace ht

extern "C" int ht_prbfit_grad(ht_prop_s* prop, const void* prb, const float* ref, void* work, void* grad, float scale,
                              void* stream) {
  using namespace ht;
  HT_REQUIRE(prop && prb && ref && work && grad, "ht_prbfit_grad: null pointer");
  int n, nz, ndist;
  prop_dims(prop, &n, &nz, &ndist);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long img = (long)nz * n, tot = img * ndist;
  float2* w = static_cast<float2*>(work);
  for (int j = 0; j < ndist; ++j) {
    const int e = prop_apply(prop, static_cast<const float2*>(prb) + j * img, w + j * img, 1, j, false, st);
    if (e != kOk) return e;
  }
  k_prbfit_resid<<<pf_grid(tot), kPfThreads, 0, st>>>(w, ref, tot);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  for (int j = 0; j < ndist; ++j) {
    const int e = prop_apply(prop, w + j * img, w + j * img, 1, j, true, st);
    if (e != kOk) return e;
  }
  return ht_axpby(grad, w, 1.0f, scale, 2 * tot, nullptr, stream);
}

extern "C" int ht_prbfit_forms(ht_prop_s* prop, const void* prb, const void* d1, const void* d2, const float* ref,
                               void* work, double* out, double scale, int hess_slots, void* stream) {
  using namespace ht;
  HT_REQUIRE(prop && prb && d1 && ref && work && out, "ht_prbfit_forms: null pointer");
  int n, nz, ndist;
  prop_dims(prop, &n, &nz, &ndist);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long img = (long)nz * n, tot = img * ndist;
  float2* Dp = static_cast<float2*>(work);
  float2* Da = Dp + tot;
  float2* Db = d2 ? Da + tot : nullptr;
  double* part = reinterpret_cast<double*>(Dp + 3 * tot);
  for (int j = 0; j < ndist; ++j) {
    int e = prop_apply(prop, static_cast<const float2*>(prb) + j * img, Dp + j * img, 1, j, false, st);
    if (e == kOk) e = prop_apply(prop, static_cast<const float2*>(d1) + j * img, Da + j * img, 1, j, false, st);
    if (e == kOk && d2) e = prop_apply(prop, static_cast<const float2*>(d2) + j * img, Db + j * img, 1, j, false, st);
    if (e != kOk) return e;
  }
  const unsigned g = pf_grid(tot);
  k_prbfit_forms<<<g, kPfThreads, 0, st>>>(Dp, Da, Db, ref, tot, part);
  count_launch();
  k_prbfit_finish<<<1, 32, 0, st>>>(part, (int)g, scale, hess_slots, out);
  count_launch();
  HT_CHECK_CUDA(cudaGetLastError());
  return kOk;
}
