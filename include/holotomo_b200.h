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

/* Number of CUDA kernels the library has launched in this process (all
 * threads); no counterpart in the reference. */
long ht_launch_count(void);

/* Page-lock [ptr, ptr + bytes) of host memory so that copies from and to it
 * run asynchronously (the host arrays Chunking.gpu_batch streams,
 * src/holotomocupy/chunking.py:100-200).  *registered = 1 if this call
 * locked it, 0 if it was page-locked already (not an error). */
int ht_host_register(void* ptr, long bytes, int* registered);
/* Undo ht_host_register. */
int ht_host_unregister(void* ptr);

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

/* ------------------------------------------------------------------------
 * Padded-grid convolution and mirror padding, for callers that work on the
 * reference's 2nz x 2n grid directly (its tests time and compare these steps).
 * Replaces the cuFFTDx convolution conv2d_create / conv2d_run /
 * conv2d_destroy (src/holotomocupy/cuda/conv2d.cu:117-159, bound in
 * conv2d_cufftdx.py:150-196) and the pad_fwd / pad_adj kernels
 * (src/holotomocupy/cuda_kernels.py:78-127, Propagation._fwd_pad/_adj_pad,
 * propagation.py:46-68).  ht_prop_D/DT do not use them.
 * --------------------------------------------------------------------- */
typedef struct ht_conv2d_s ht_conv2d_s;

/* A convolution of [rows, cols] complex64 images; rows, cols: 2^a 3^b from
 * 18 to 4096.  The handle holds only shared twiddle tables (no workspace). */
int ht_conv2d_create(int rows, int cols, ht_conv2d_s** out);
int ht_conv2d_destroy(ht_conv2d_s* h);
/* y[b] = IFFT2(FFT2(x[b]) * H) for b < batch, the inverse unnormalised
 * (rows*cols times the normalised one, as conv2d_run); x, y [batch, rows,
 * cols], H [rows, cols] complex64; y may alias x. */
int ht_conv2d_run(ht_conv2d_s* h, const void* x, const void* H, void* y, long batch, void* stream);

/* fpad[batch, 2nz, 2n] = the half-sample-symmetric (mirror) extension of
 * f[batch, nz, n] centred on the padded grid (pad_fwd); n, nz even. */
int ht_pad_mirror(const void* f, void* fpad, long batch, int nz, int n, void* stream);
/* f[batch, nz, n] = the adjoint of ht_pad_mirror: each sample sums the four
 * padded samples that copy it (pad_adj). */
int ht_pad_fold(const void* fpad, void* f, long batch, int nz, int n, void* stream);

/* ------------------------------------------------------------------------
 * USFFT Radon transform.  Replaces Tomo.__init__/R/RT
 * (src/holotomocupy/tomo.py:12-54, 56-86, 88-116) and the gather kernel
 * (src/holotomocupy/cuda_kernels.py:3-76).
 * --------------------------------------------------------------------- */
typedef struct ht_tomo_s ht_tomo_s;

/* n: object width (= detector width); nz: slice capacity of one call;
 * theta_host: host float32 [ntheta]; phi_host: host float32 [n, n], the
 * reference's deapodisation factor already multiplied by the support mask
 * and 1/(n sqrt(n ntheta)) (tomo.py:19-21, 34-47).  The handle owns a
 * workspace of nz*(6n^2) + ntheta*nz*n complex64 samples. */
int ht_tomo_create(int n, int nz, int ntheta, const float* theta_host, const float* phi_host, ht_tomo_s** out);
int ht_tomo_destroy(ht_tomo_s* t);

/* sino[ntheta, nz, n] = R(obj[nz, n, n]), complex64 (tomo.py:56-86). */
int ht_tomo_R(ht_tomo_s* t, const void* obj, void* sino, int nz, void* stream);

/* obj[nz, n, n] = R^T(sino[ntheta, nz, n]), complex64 (tomo.py:88-116). */
int ht_tomo_RT(ht_tomo_s* t, const void* sino, void* obj, int nz, void* stream);
/* R followed by the detector-axis half of the B-spline prefilter, and R^T
 * preceded by it: Cx(R obj) and R^T(Cx sino), Cx the circulant filter with
 * symbol 1 / (4 + 2 cos 2 pi k / n) along the last axis (shift.py:74-82, its
 * row factor), applied in R's own detector spectrum at no extra pass.  With
 * ht_shift_coeff_z on the volume they give coeff(R obj) = Cx R Cz obj and
 * R^T coeff(sino) = Cz R^T Cx sino (the z factor commutes with R). */
int ht_tomo_R_coeffx(ht_tomo_s* t, const void* obj, void* sino, int nz, void* stream);
/* ... and obj = scale * R^T(Cx sino): the BH variable scaling rho of the
 * object gradient (rec_mpi.py:345) applied in the same pass. */
int ht_tomo_RT_coeffx(ht_tomo_s* t, const void* sino, void* obj, int nz, float scale, void* stream);
/* R and R^T of a slab of nz object slices inside a taller sinogram (object
 * slabs processed in turn when the handle's workspace holds fewer slices
 * than the volume): the slab's row z of angle th is at sino[(th * ldz + z) *
 * n], sino offset to the slab's first row, ldz >= nz the sinogram's rows per
 * angle.  coeffx = 1: with the detector-axis prefilter of the _coeffx forms;
 * scale multiplies R^T's result. */
int ht_tomo_R_slab(ht_tomo_s* t, const void* obj, void* sino, int nz, int ldz, int coeffx, void* stream);
int ht_tomo_RT_slab(ht_tomo_s* t, const void* sino, void* obj, int nz, int ldz, int coeffx, float scale,
                    void* stream);

/* ------------------------------------------------------------------------
 * Cubic B-spline shift family.  Replaces Shift.__init__/coeff/S/Sadj/
 * dcurlySc/dcurlySadjc/d2curlySc (src/holotomocupy/shift.py:18-48, 74-82,
 * 102-122, 170-221) and the kernels s/sf, ds/dsf, d2s/d2sf, dsadj/dsadjf
 * (src/holotomocupy/cuda_kernels.py:161-290, 377-843).
 * Shapes: coefficients [batch, nzpsi, npsi]; shifted images [batch, nz, n];
 * r, dr: float32 [batch, 2] as (y, x) shifts in pixels; mag: float32 [batch].
 * is_complex = 1: complex64 elements; 0: float32 elements.
 * --------------------------------------------------------------------- */
typedef struct ht_shift_s ht_shift_s;

int ht_shift_create(int n, int npsi, int nz, int nzpsi, int is_complex, ht_shift_s** out);
int ht_shift_destroy(ht_shift_s* s);

/* out = ifft2(fft2(psi) / B3): the B-spline prefilter (shift.py:74-82);
 * complex64 [batch, nzpsi, npsi]; out may alias psi. */
int ht_shift_coeff(ht_shift_s* s, const void* psi, void* out, long batch, void* stream);
/* The z-axis half of the prefilter (the column factor of shift.py:74-82):
 * out = Cz in for in, out [nzpsi, ncols] complex64 (a volume [nzpsi, ny, nx]
 * has ncols = ny nx); out may alias in. */
int ht_shift_coeff_z(ht_shift_s* s, const void* in, void* out, long ncols, void* stream);

/* out = ifft2(fft2(psi) * (symy (x) symx)): a separable periodic filter with
 * caller-given device symbols symx [npsi], symy [nzpsi] in FFT order, each
 * carrying its 1/N.  Shift.coeffback (shift.py:84-96) is this filter with
 * the stretched B-spline's inverse symbol; complex64 [batch, nzpsi, npsi],
 * out may alias psi. */
int ht_shift_filter(ht_shift_s* s, const void* psi, void* out, long batch, const float* symx, const float* symy,
                    void* stream);

/* out = Sback_{r,mag}(g) (shift.py:138-148; sback, cuda_kernels.py:294-370):
 * the back-projection of detector images g [batch, nz, n] complex64 onto the
 * coefficient grid [batch, nzpsi, npsi] complex64 with the B-spline stretched
 * by mag (nmag = 1: one magnification for every image; nmag = batch: one
 * each); every cell of out is written (a deterministic gather, no atomics). */
int ht_shift_Sback(ht_shift_s* s, const void* g, const float* r, const float* mag, int nmag, void* out, long batch,
                   void* stream);

/* out = S_{r,mag}(c) (shift.py:102-111; cuda_kernels.py:161-227). */
int ht_shift_S(ht_shift_s* s, const void* c, const float* r, const float* mag, void* out, long batch, void* stream);

/* out = S_{r,mag}^T(g) (shift.py:113-122), deterministic gather form. */
int ht_shift_Sadj(ht_shift_s* s, const void* g, const float* r, const float* mag, void* out, long batch,
                  void* stream);

/* First derivative: S(c1) - (dS/dr . dr)(c) (shift.py:170-183; cuda_kernels.py:547-617). */
int ht_shift_dS(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* c1, const float* dr,
                void* out, long batch, void* stream);

/* Second-order term with the reference's pairing of (c1, dr1) and (c2, dr2)
 * (shift.py:206-221; cuda_kernels.py:377-459). */
int ht_shift_d2S(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* c1, const float* dr1,
                 const void* c2, const float* dr2, void* out, long batch, void* stream);

/* Adjoint of the derivative (shift.py:185-204; cuda_kernels.py:690-766):
 * out1 = S^T(g) [batch, nzpsi, npsi]; out2 = double [batch, 2] with
 * out2[b,0] = Re<g, -phi'_y phi_x c>, out2[b,1] = Re<g, -phi'_x phi_y c>,
 * reduced in double precision (the reference returns float32). */
int ht_shift_dSadj(ht_shift_s* s, const void* c, const float* r, const float* mag, const void* g, void* out1,
                   double* out2, long batch, void* stream);

/* ------------------------------------------------------------------------
 * Fused BH data-fidelity cascade.  Replaces Rec.gradients_cascade,
 * Rec.hessian_cascade and the forward model of Rec.min/gen_sqrt_data
 * (src/holotomocupy/rec_mpi.py:250-353, 498-507, 517-813, 815-835,
 * 882-897) with its F0..F3 / dF / d2F_dF / gF chain.
 * Shapes (nimg = ntheta*ndist): c [ntheta, nzobj, nobj] B-spline
 * coefficients of proj (complex64, or float32 when is_complex = 0);
 * pos [ntheta, ndist, 2] float32 (y, x); mag [ntheta, ndist] float32;
 * prb [ndist, nz, n] complex64; data [ntheta, ndist, nz, n] float32
 * amplitudes.  The handle owns 4*nimg*nz*n complex64 samples of workspace:
 * caches of the last gradient call that ht_rec_hessian reads, so call
 * ht_rec_gradient first with the same state.
 * --------------------------------------------------------------------- */
typedef struct ht_rec_s ht_rec_s;

int ht_rec_create(int n, int nz, int nobj, int nzobj, int ntheta, int ndist, int is_complex, ht_prop_s* prop,
                  ht_rec_s** out);
int ht_rec_destroy(ht_rec_s* r);

/* Forward model.  With amp != NULL: amp[ntheta, ndist, nz, n] = |x0|
 * (gen_sqrt_data, rec_mpi.py:882-897).  Otherwise *fval (device double) =
 * sum (|x0| - data)^2; divided by N = ntheta*ndist*nz*n it is F0 of min
 * (rec_mpi.py:517-527, 815-835). */
int ht_rec_forward(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb, const float* data,
                   float* amp, double* fval, void* stream);

/* A handle created for an angle chunk of a larger problem: N of the
 * objective's 2/N (rec_mpi.py:569, 91) becomes the whole problem's
 * ntheta*ndist*nz*n.  With it, ht_rec_gradient / ht_rec_hessian called on the
 * chunks in turn (pointers offset to the chunk's angles, accumulate = 1 after
 * the first) give the whole problem's sums.  A chunk's Hessian reads the
 * caches of that chunk's gradient call, so a chunked Hessian evaluation
 * repeats each chunk's gradient call before its Hessian call. */
int ht_rec_set_data_size(ht_rec_s* r, double ndata);

/* shared = 1: the coefficient arguments (c, and cy, cz of ht_rec_hessian) are
 * one [nzobj, nobj] array for every angle, and ht_rec_gradient's gc is its
 * gradient summed over all images, [nzobj, nobj].  Near-field ptychography
 * (RecNFP, src/holotomocupy/rec_nfp_mpi.py:20-469) scans one projection over
 * ntheta positions at one distance; the reference tiles the coefficients over
 * the positions (rec_nfp_mpi.py:353-357) and sums the per-position adjoints
 * (:393-405). */
int ht_rec_set_shared_coefficients(ht_rec_s* r, int shared);

/* Gradient of the data term (gF0..gF3, rec_mpi.py:327-353, 562-813):
 * gc [ntheta, nzobj, nobj] = sum_k S_k^T(Y22) (unscaled; apply coeff() for
 * the proj gradient), gpos [ntheta, ndist, 2] float32 times scale_pos,
 * gprb [ndist, nz, n] complex64 times scale_prb (the variable scalings
 * rho_sq of rec_mpi.py:345-347; 1 for the plain gradient), *fval (device
 * double) = sum (|x0| - data)^2 at the same point.  accumulate = 1: gprb and
 * *fval are added to (an angle chunk after the first; gc and gpos cover only
 * the chunk's angles and are written). */
int ht_rec_gradient(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb,
                    const float* data, void* gc, float* gpos, void* gprb, double* fval, float scale_pos,
                    float scale_prb, int accumulate, void* stream);

/* Hessian forms at the state of the last ht_rec_gradient call
 * (hessian_cascade, rec_mpi.py:250-303) for directions y (and z when
 * ndir = 2), each given as (coefficients of its proj, its pos, its prb).
 * out (device double[4]) = {H(y,y), H(y,z) as the reference evaluates it
 * (its d2s pairs c_y with r_y and c_z with r_z), H(z,z), the symmetric
 * H(y,z)}; accumulate = 1 adds to out (an angle chunk after the first). */
int ht_rec_hessian(ht_rec_s* r, const void* c, const float* pos, const float* mag, const void* prb,
                   const float* data, int ndir, const void* cy, const float* posy, const void* prby, const void* cz,
                   const float* posz, const void* prbz, double* out, int accumulate, void* stream);

/* ------------------------------------------------------------------------
 * BLAS-1 on float32 vectors (complex64 arrays as interleaved pairs, n =
 * number of floats), inner products accumulated in double.  Replaces
 * Chunking.linear_batch / linear_redot_batch / redot_batch
 * (src/holotomocupy/chunking.py:235-290) and utils.redot (utils.py:100-103).
 * --------------------------------------------------------------------- */
/* x = a*x + b*y; if dot != NULL: *dot += sum(y * x_new) (device double). */
int ht_axpby(void* x, const void* y, float a, float b, long n, double* dot, void* stream);
/* *dot += sum(x * y) (device double). */
int ht_dot(const void* x, const void* y, long n, double* dot, void* stream);
/* x = a*x + b*y with a = (float)(*A) * sa and b = (float)(*B) * sb read on
 * the device when the stream reaches the call (A or B NULL: the factor
 * alone); dot as in ht_axpby.  The BH direction and variable updates
 * (rec_mpi.py:196-218) with step sizes that never visit the host. */
int ht_axpby_dev(void* x, const void* y, const double* A, float sa, const double* B, float sb, long n, double* dot,
                 void* stream);
/* BH step sizes on the device (rec_mpi.py:180-218, with the forms of
 * ht_rec_hessian in H[4] and dots[3] = <eta,grad> of obj, pos, prb).
 * phase 0: scal[0] = beta = first ? 0 : H[1]/H[2]; dots[0..2] = 0 if dots
 *          != NULL (the direction updates then accumulate into them).
 * phase 1: scal[1] = alpha = -(dots[0]/rho_obj + dots[1]/rho_pos + dots[2]/rho_prb)
 *          / (first ? H[0] : beta^2 H[2] - 2 beta H[3] + H[0]);
 *          if hist: (alpha, beta) goes to hist[2*(*count)] while *count < cap,
 *          and *count is incremented (device int). */
int ht_bh_scalars(const double* H, double* dots, int first, int phase, double rho_obj, double rho_pos,
                  double rho_prb, double* scal, double* hist, int cap, int* count, void* stream);

/* The objective sum (|x0| - data)^2 of ht_rec_forward, without allocating.
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (their memory belongs to another allocator, or they must not call
 * cudaMalloc/cudaFree because those can synchronise the device): needs only
 * the propagator handle (created once at set-up) and the inputs, and works
 * in one fixed 32 MiB device array that every GPU loading the library holds
 * until exit.  Angles are processed in chunks that fit it; one angle needs
 * ndist*nz*n*8 + ndist*(nz+1)*8 bytes, and larger sizes are rejected
 * (status 1).  The sum is reduced in a fixed order (bitwise reproducible).  The first
 * call on a device looks up the array's device address: make it before any
 * stream capture.  All calls share the array, so calls that overlap on the
 * GPU race; run them in one stream. */
int ht_rec_objective_noalloc(ht_prop_s* prop, int nobj, int nzobj, int ntheta, int is_complex, const void* c,
                             const float* pos, const float* mag, const void* prb, const float* data, double* fval,
                             void* stream);

/* ------------------------------------------------------------------------
 * Probe-fit regulariser lam |||D prb| - ref||^2 / (ndist nz n) on the device.
 * Replaces Rec.gradient_prbfit and Rec.hessian_prbfit
 * (src/holotomocupy/rec_mpi.py:365-398), whose host-side sums keep a BH
 * iteration with the term out of a CUDA graph.  prb, d1, d2: complex64
 * [ndist, nz, n]; ref: float32 [ndist, nz, n] (|D prb_true|, gen_sqrt_ref).
 * --------------------------------------------------------------------- */
/* grad += scale * D^H(2 (D prb - ref D prb / |D prb|)) per distance
 * (scale = lam / (ndist nz n) times the variable scaling rho_prb);
 * work: ndist*nz*n complex64. */
int ht_prbfit_grad(ht_prop_s* prop, const void* prb, const float* ref, void* work, void* grad, float scale,
                   void* stream);
/* The forms f(u, w) = 2 scale sum (1 - ref/|p|) Re(u conj w) + ref/|p| Re(conj(l) u) Re(conj(l) w),
 * p = D prb, l = p/|p|, u = D d1, w = D d2, for the pairs (d1,d1), (d1,d2),
 * (d2,d2) (d2 = NULL: the first only), reduced in FP64 in a fixed order.
 * hess_slots = 0: out[0..2] = the three forms; hess_slots = 1: out[0] +=
 * f(d1,d1), out[1] += f(d1,d2), out[2] += f(d2,d2), out[3] += f(d1,d2) (the
 * slots of ht_rec_hessian).  work: 3*ndist*nz*n complex64 plus 32 KiB. */
int ht_prbfit_forms(ht_prop_s* prop, const void* prb, const void* d1, const void* d2, const float* ref, void* work,
                    double* out, double scale, int hess_slots, void* stream);

/* ------------------------------------------------------------------------
 * 3-D Laplacian regulariser (rec_mpi.py:402-496).  Arrays [nz, ny, nx],
 * complex64 (is_complex) or float32; work: (nz + 2) * ny * nx elements of the
 * same type, then, from the next 16-byte boundary, 64 KiB for the per-block
 * partial sums of the forms and the energy (added in a fixed order).  L: the 7-point Laplacian, periodic in y and x, of the object
 * zero-padded in z; B = L o L with the inner L also on the ghost slice at each
 * end, as the reference evaluates it.
 * --------------------------------------------------------------------- */
/* g += scale * B u  (gradient_laplacian, rec_mpi.py:419-442) */
int ht_laplacian_grad(const void* u, void* g, int nz, int ny, int nx, int is_complex, float scale, void* work,
                      void* stream);
/* *out += scale * Re<y, B z>, and *out2 += scale * Re<y2, B z> if y2 != NULL (device
 * doubles; hessian_laplacian, rec_mpi.py:444-470) */
int ht_laplacian_dot(const void* y, const void* z, int nz, int ny, int nx, int is_complex, double scale, void* work,
                     double* out, const void* y2, double* out2, void* stream);
/* *out += scale * sum over the object slices of |L u|^2  (_lap_energy_local, rec_mpi.py:472-496) */
int ht_laplacian_energy(const void* u, int nz, int ny, int nx, int is_complex, double scale, void* work, double* out,
                        void* stream);

/* Row filter: out[r] = IFFT(sym * FFT(in[r])) for each of nrows rows of
 * length N (complex64); sym: device float32 [N] in FFT order, carrying the
 * 1/N of the inverse transform.  Serves Tomo._filter_sino
 * (src/holotomocupy/tomo.py:118-161). */
int ht_filter_rows(int N, const void* in, void* out, long nrows, const float* sym, void* stream);

/* ------------------------------------------------------------------------
 * CUDA graphs of a stream's work (the reference launches every kernel from
 * Python each iteration; no counterpart).  ht_graph_begin starts recording
 * the work issued to `stream` (a non-default stream, relaxed capture mode); nothing
 * runs until the graph is launched.  ht_graph_end ends the recording and
 * returns an executable graph in *exec; ht_graph_launch runs it on a stream;
 * ht_graph_destroy frees it.  Everything recorded must already have run
 * once on this device (so launch attributes and tables exist).
 * --------------------------------------------------------------------- */
int ht_graph_begin(void* stream);
int ht_graph_end(void* stream, void** exec);
int ht_graph_launch(void* exec, void* stream);
int ht_graph_destroy(void* exec);

/* Per-kernel CUDA-event timers (instrumentation; no counterpart).  Arming a
 * kernel's timer (names: k_casc_fwd, k_casc_resid, k_casc_resid_f,
 * k_casc_adj, k_casc_hess_fwd, k_casc_hess_q, k_dct_cols, k_tgather,
 * k_tcell) clears its record; while armed, every launch of it outside graph
 * capture is bracketed by an event pair on its stream.  ht_ktimer_read
 * waits for the recorded launches and returns their summed time, their
 * count and their summed work units (images for the cascade and column
 * kernels, slices for k_tgather and k_tcell). */
int ht_ktimer_arm(const char* name, int on);
int ht_ktimer_read(const char* name, double* total_ms, long* launches, double* units);

#ifdef __cplusplus
}
#endif

#endif /* HOLOTOMO_B200_H */
