// Internal declarations shared by the operator translation units.
#pragma once
#include <cuda_runtime.h>

#include "../../include/holotomo_b200.h"

namespace ht {
cudaError_t dct_rows(int N, bool inverse, const float2* in, float2* out, long nrows, const float2* tw4,
                     cudaStream_t st);
cudaError_t dct_cols(int NZ, bool conj, float2* data, long nimg, int n, const float2* H, int ntab,
                     const float2* tw4, cudaStream_t st);
int prop_apply(ht_prop_s* p, const void* in, void* out, long batch, int j, bool adjoint, cudaStream_t st);
void prop_dims(const ht_prop_s* p, int* n, int* nz, int* ndist);
void prop_tables(const ht_prop_s* p, const float2** hw, const float2** twn, const float2** twz);
}  // namespace ht

namespace ht {
cudaError_t symbol_rows(int N, const float2* in, float2* out, long nrows, const float* sym, const float2* tw,
                        cudaStream_t st);
cudaError_t symbol_cols(int N, const float2* in, float2* out, long nimg, int ncols, const float* sym,
                        const float2* tw, cudaStream_t st);
}  // namespace ht
