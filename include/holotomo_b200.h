/*
 * holotomo_b200 — C ABI of the B200 operator chain for X-ray holotomography.
 *
 * Every function is stream-ordered on the CUDA stream passed as `stream`
 * (a cudaStream_t, NULL = legacy default stream) and returns an int status:
 *   0 = ok, 1 = bad argument, 2 = CUDA error, 3 = unsupported size.
 * ht_last_error() returns the message of the calling thread's last failure.
 * All data pointers are device pointers owned by the caller unless a comment
 * says "host".  Complex arrays are interleaved complex64 (float re, float im),
 * C-contiguous.  Handles own their constant tables and, where stated, a
 * workspace; one handle must not be used from two streams at the same time
 * (create one handle per stream instead).
 *
 * Each declaration names the reference interface it replaces
 * (nikitinvv/holotomocupy, paths relative to its repository root).
 */
#ifndef HOLOTOMO_B200_H
#define HOLOTOMO_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Library version (major*10000 + minor*100 + patch). */
int ht_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* ht_last_error(void);

/* ------------------------------------------------------------------------
 * Fresnel propagator.  Replaces Propagation.__init__/D/DT
 * (src/holotomocupy/propagation.py:14-44, 70-89, 91-112) and the cuFFTDx
 * convolution C ABI conv2d_create/conv2d_run/conv2d_destroy
 * (src/holotomocupy/cuda/conv2d.cu:117-159).
 * --------------------------------------------------------------------- */
typedef struct ht_prop_s ht_prop_s;

/* fker_host: host complex64 [ndist, 2*nz, 2*n], the reference's Fresnel
 * table fker[j] = exp(-i pi lambda z_j (fx^2+fy^2)) / (4 n nz) on the padded
 * fftfreq grid (propagation.py:20-28).  n, nz: detector width and height. */
int ht_prop_create(int n, int nz, int ndist, const void* fker_host, ht_prop_s** out);
int ht_prop_destroy(ht_prop_s* p);

/* out[b] = D_j(in[b]) for b < batch; in, out: complex64 [batch, nz, n];
 * out may alias in.  No workspace. (propagation.py:70-89) */
int ht_prop_D(ht_prop_s* p, const void* in, void* out, long batch, int j, void* stream);

/* out[b] = D_j^H(in[b]) (propagation.py:91-112); same layout rules as D. */
int ht_prop_DT(ht_prop_s* p, const void* in, void* out, long batch, int j, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* HOLOTOMO_B200_H */
