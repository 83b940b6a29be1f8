/*
 * model_mosaic_b200 C-ABI: the forward-model hot path of model_mosaic on one
 * B200 (sm_100a).  Plain pointers and sizes only; every compute call takes
 * device pointers and a cudaStream_t passed as `void*` (NULL = legacy default
 * stream) and returns MM_OK (0) or a negative MM_E* status.  No call aborts
 * the process; the text of the last error on the calling thread is returned
 * by mm_last_error().  A handle is not thread-safe: use one per host thread.
 * Handles own their workspace; the caller owns every array it passes.
 *
 * Array layouts are the reference's (C order):
 *   obj  (nz, n, n)        float32          TomoReal.R input / RT output
 *   sino (ntheta, nz, n)   float32|complex64 TomoReal.R output / RT input
 *   psi  (ntheta, nz, n)   complex64        Propagation.D input / output
 */
#ifndef MODEL_MOSAIC_B200_MOSAIC_H
#define MODEL_MOSAIC_B200_MOSAIC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MM_OK         0
#define MM_EINVAL    -1   /* bad argument / unsupported size */
#define MM_ENOMEM    -2   /* device allocation failed */
#define MM_ECUDA     -3   /* CUDA runtime error */
#define MM_ECUFFT    -4   /* cuFFT error */
#define MM_ETIMEOUT  -5   /* a bounded device wait gave up */

#define MM_F32  0
#define MM_C64  1
#define MM_BF16 2   /* bfloat16 storage; arithmetic stays float32 */

typedef struct mm_tomo mm_tomo;
typedef struct mm_prop mm_prop;
typedef struct mm_fbp mm_fbp;
typedef struct mm_pgn mm_pgn;

/* USFFT options.  Zero-initialised fields take the reference defaults
 * (processing/tomo.py:39-42): eps = 1e-3, m from eps (m = 4), oversampling 2.
 * The adjoint's scatter table is built per block of angles, sized by the
 * free device memory; blocks after the first add into the first block's
 * result.  When all blocks do not fit at once (very large n and angle
 * counts, e.g. n = 24576 with 18432 angles) they are rebuilt one at a time
 * at every RT call. */
typedef struct mm_tomo_opts {
    double eps;        /* Gaussian accuracy; <= 0 -> 1e-3 */
    int    m;          /* half-width override; <= 0 -> from eps (reference formula) */
    int    clamp_xy;   /* 1: clamp sample coordinates to [-1/2, 1/2 - 1e-5] in R as
                          TomoLargeReal's gather does (processing/kernels.py:478-481) */
    int    compensated;  /* 1: Kahan-compensated sums in the adjoint scatter */
    int    max_table_angles;  /* > 0: at most this many angles per block of the adjoint's
                                 scatter table (0: as many as device memory allows) */
    int    reserved[3];
} mm_tomo_opts;

/* Library and error reporting. */
int         mm_version(void);
int         mm_last_error(char* buf, size_t len);  /* copies the message, returns its length */

/* Caller-array checks, process-wide, off by default (also on with the
 * environment variable MM_BOUNDS_CHECK=1).  When on, every compute call first
 * checks each array argument: device memory of the current device (or mapped
 * pinned host memory), and the bytes the call reads or writes lie inside one
 * allocation (for arrays carved out of a larger allocation, inside that
 * allocation).  A failure returns MM_EINVAL naming the argument, before
 * anything is launched.  Costs one pointer query per array per call. */
int         mm_set_bounds_check(int on);
int         mm_get_bounds_check(void);
/* The same check on one array, whatever the switch: MM_OK when [p, p + bytes)
 * is device (or mapped pinned host) memory of the current device inside one
 * allocation, else MM_EINVAL with the reason in mm_last_error(). */
int         mm_check_array(const void* p, size_t bytes);

/* ---- USFFT Radon pair ---------------------------------------------------
 * mm_tomo_create replaces TomoReal.__init__(n, nz, theta)
 *   (processing/tomo.py:30-88) and TomoLargeReal.__init__(n, theta, chunk_xy)
 *   (processing/tomo_large.py:72-148).  theta_host: ntheta float32 radians.
 *   opts may be NULL (reference defaults).  n must be even, 8 <= n <= 32768. */
int mm_tomo_create(int n, int nz, int ntheta, const float* theta_host,
                   const mm_tomo_opts* opts, mm_tomo** out);
/* Replaces TomoReal.free (processing/tomo.py:109-119) / TomoLargeReal.free. */
int mm_tomo_destroy(mm_tomo* h);

/* Replaces TomoReal.R (processing/tomo.py:121-151) and TomoLargeReal.R
 *   (processing/tomo_large.py:344-368): obj (nz, n, n) f32 -> sino
 *   (ntheta, nz, n) f32, for 1 <= nz <= the handle's nz.  Device pointers. */
int mm_tomo_R(mm_tomo* h, const float* obj, float* sino, int nz, void* stream);
/* mm_tomo_R with a storage type per array (MM_F32 or MM_BF16 each): bfloat16
 *   storage of the volume and/or the sinogram, float32 arithmetic.  No
 *   reference counterpart (the reference stores float32 only). */
int mm_tomo_R_ex(mm_tomo* h, const void* obj, int obj_dtype, void* sino, int sino_dtype, int nz,
                 void* stream);

/* Replaces TomoReal.RT (processing/tomo.py:153-188) and TomoLargeReal.RT
 *   (processing/tomo_large.py:582-630): sino (ntheta, nz, n) of `dtype`
 *   (MM_F32, MM_C64 or MM_BF16) -> obj (nz, n, n) of the same dtype (real
 *   part only for real input, as the reference).  Deterministic: no float
 *   atomics. */
int mm_tomo_RT(mm_tomo* h, const void* sino, int dtype, void* obj, int nz, void* stream);

/* Builds the adjoint's static scatter table now instead of on the first RT
 * call (the reference defers its RT buffers the same way, tomo.py:90-107). */
int mm_tomo_prepare_rt(mm_tomo* h, void* stream);

/* Bytes of device workspace the handle holds now. */
size_t mm_tomo_workspace_bytes(const mm_tomo* h);

/* Per-stage CUDA-event timing (tracing; no reference counterpart -- the
 * reference times whole stages with perf_counter, step2_radon.py:186-197).
 * set_timing(1) resets and starts recording events around every stage on the
 * call's stream; get_timing waits for them and returns, for up to nstages
 * stages, the summed milliseconds and call counts, and the number of this
 * library's own kernel launches since timing was switched on.
 * Tomo stages: 0 pad+phi, 1 x-R2C, 2 transpose in, 3 y-FFT, 4 gather,
 *   5 r-C2R (+ slice crop), 6 r-R2C (RT), 7 scatter, 8 y-IFFT, 9 transpose out,
 *   10 x-C2R, 11 crop*phi, 12 scatter-table build, 13 complex-RT prologue. */
int mm_tomo_set_timing(mm_tomo* h, int on);
int mm_tomo_get_timing(mm_tomo* h, double* ms, long long* calls, int nstages, long long* kernels);

/* ---- Fresnel propagator -------------------------------------------------
 * mm_prop_create replaces Propagation.__init__(n, nz, ntheta, ndist,
 *   wavelength, voxelsize, distance) (processing/propagation.py:18-35) and
 *   PropagationLarge.__init__ (processing/propagation_large.py:55-94).
 *   Any n, nz in [2, 32768]: powers of two up to 2048 run the fused
 *   two-pass kernels, other sizes the general path (cuFFT 2-D transforms
 *   between reordering kernels). */
int mm_prop_create(int n, int nz, int ntheta, int ndist, double wavelength,
                   double voxelsize, const double* distance_host, mm_prop** out);
int mm_prop_destroy(mm_prop* h);

/* Replaces Propagation.D (processing/propagation.py:47-64) and
 *   PropagationLarge.D (processing/propagation_large.py:202-236):
 *   psi (ntheta, nz, n) c64 -> out (ntheta, nz, n) c64, distance index j.
 *   psi and out may alias. */
int mm_prop_D(mm_prop* h, const void* psi, void* out, int ntheta, int j, void* stream);

/* Adjoint of D (no reference counterpart: the reference ships only D,
 *   processing/propagation_large.py:15).  Same layouts as mm_prop_D. */
int mm_prop_DT(mm_prop* h, const void* g, void* out, int ntheta, int j, void* stream);

/* step3_propagation.py:218-225 fused: proj (ntheta, nz, n) f32 ->
 *   psi = exp(-p*s/beta_r) (cos p*s, sin p*s) with s = inv_norm,
 *   1/beta_r = inv_beta_ratio (_psi_from_proj, :94-103) -> D -> |.|^2
 *   (_abs2_c64_to_f32, :105-110) -> intensity (ntheta, nz, n) f32. */
int mm_prop_intensity(mm_prop* h, const float* proj, float inv_norm, float inv_beta_ratio,
                      float* intensity, int ntheta, int j, void* stream);

/* Differentiable forward model data = |D psi|^2, psi = exp(-p s/beta_r)(cos p s, sin p s),
 * p = R delta (no reference counterpart: the reference composes R, psi, D and |.|^2 only
 * across step2 -> disk -> step3 and has no adjoint of D).  With the L2 loss
 * L = sum (|D psi|^2 - data)^2:
 *   mm_prop_grad_forward: gu = 4 (|D psi|^2 - data) D psi (complex, (ntheta, nz, n)) and
 *     per-block sums of (|D psi|^2 - data)^2 in partials[0 .. mm_prop_grad_partials());
 *   mm_prop_grad_backward: gp = dL/dp = s Re(conj(D^H gu) (i - 1/beta_r) psi), float.
 * dL/d delta is then mm_tomo_RT(gp).  inv_norm = s, inv_beta_ratio = 1/beta_r. */
long mm_prop_grad_partials(mm_prop* h, int ntheta);
int mm_prop_grad_forward(mm_prop* h, const float* proj, const float* data, float inv_norm,
                         float inv_beta_ratio, void* gu, float* partials, int ntheta, int j, void* stream);
int mm_prop_grad_backward(mm_prop* h, const void* gu, const float* proj, float inv_norm,
                          float inv_beta_ratio, float* gp, int ntheta, int j, void* stream);

/* Allocation-free Fresnel D for callers that cannot allocate device memory
 *   while they run (their GPU memory is reserved up front by their own pool
 *   allocator, so a cudaMalloc mid-run fails or stalls other work).  No
 *   counterpart in the reference.  Same operator and layouts as mm_prop_D for
 *   one distance, without a handle, for n and nz powers of two in [2, 2048]
 *   (the fused two-pass kernels; mm_prop_D also takes other sizes): the
 *   chirp/twiddle tables and the intermediate live in one static 64 MiB
 *   device array per GPU, so (ntheta*nz*n + 8*(n+nz)) * 8 bytes must fit in
 *   64 MiB (MM_EINVAL otherwise).  CUDA loads device code lazily, so the
 *   first call on each device is what loads this code and takes the 64 MiB
 *   (kept until the process exits) and resolves the array's address: make
 *   one call on each device before reserving a device memory pool and before
 *   any stream capture.  Calls share the array: calls that overlap on the GPU
 *   race and must be ordered by the caller. */
int mm_prop_D_noalloc(int n, int nz, int ntheta, double wavelength, double voxelsize, double distance,
                      const void* psi, void* out, void* stream);

/* Stage timing as for mm_tomo_*_timing.  Stages: 0 y-pass (columns), 1 x-pass (rows). */
int mm_prop_set_timing(mm_prop* h, int on);
int mm_prop_get_timing(mm_prop* h, double* ms, long long* calls, int nstages, long long* kernels);

/* ---- FBP filter (step8_fbp path) ----------------------------------------
 * mm_fbp_create replaces FBPFilter.__init__(n, batch_chunk)
 *   (processing/fbp_filter.py:41-47).  Rows with 4n a power of two in
 *   [16, 8192] are filtered in place by one fused kernel without scratch;
 *   other n use cuFFT over batch_chunk rows at a time. */
int mm_fbp_create(int n, int batch_chunk, mm_fbp** out);
int mm_fbp_destroy(mm_fbp* h);
/* Replaces FBPFilter.filter(sino, w) (processing/fbp_filter.py:128-192): the
 *   `rows` rows of n float32 samples at `sino` (device) filtered in place with
 *   the device weights w (2n + 1) of FBPFilter.calc_filter (:49-88, host-side
 *   FP64 arithmetic, computed by the caller as the reference does):
 *   edge-replicated padding to 4n, spectrum times w, inverse, centre n kept. */
int mm_fbp_filter(mm_fbp* h, float* sino, long rows, const float* w, void* stream);
size_t mm_fbp_workspace_bytes(const mm_fbp* h);

/* ---- Paganin phase retrieval (step7_paganin path) ------------------------
 * mm_pgn_create replaces Paganin.__init__(n, nz, ntheta, wavelength,
 *   voxelsize, distance, alpha) (processing/paganin.py:38-62): filt_host is
 *   the (nz, n/2 + 1) float32 filter table alpha / (lambda z |k|^2/(4 pi) +
 *   alpha) on the (fftfreq(nz), rfftfreq(n)) grid, computed by the caller as
 *   the reference does (:46-53).  n, nz powers of two up to 4096 run three
 *   fused passes; other sizes cuFFT R2C/C2R over ntheta frames. */
int mm_pgn_create(int n, int nz, int ntheta, const float* filt_host, mm_pgn** out);
int mm_pgn_destroy(mm_pgn* h);
/* Replaces Paganin.retrieve (processing/paganin.py:64-91): frames (<= ntheta)
 *   of (nz, n) float32 intensity -> -log(clip(irfft2(H rfft2(I)), 1e-6)),
 *   same shape, into `phase` (device). */
int mm_pgn_retrieve(mm_pgn* h, const float* intensity, float* phase, int frames, void* stream);
size_t mm_pgn_workspace_bytes(const mm_pgn* h);

/* ---- Mosaic tiles (step4_extract / step6_stitch path) --------------------
 * mm_mosaic_create takes the placements of read_placements
 *   (step4_extract.py:52-118) for a big projection of (nz, n) pixels:
 *   rects holds n_place rows of 8 ints (r_lo_dir, r_hi_dir, c_lo_dir,
 *   c_hi_dir, r_lo_mir, r_hi_mir, c_lo_mir, c_hi_mir), in placement order;
 *   overlap is the positions header's OVERLAP, the tent-weight cap
 *   (step6_stitch.py:70-81).  Footprints must lie inside (nz, n), direct and
 *   mirror share rows and width; at most 240 placements and at most 32
 *   footprints over one pixel. */
typedef struct mm_mosaic mm_mosaic;
int mm_mosaic_create(int nz, int n, int n_place, const int* rects, int overlap, mm_mosaic** out);
int mm_mosaic_destroy(mm_mosaic* h);
/* Replaces the crop loop of step4_extract.py:176-192 for nth angles: proj
 *   (nth, nz, n) float32 device; dir[p] and mir[p] (host arrays of n_place
 *   device pointers) each receive (nth, h_p, w_p) frames: the direct crop and
 *   the h-flipped mirror crop. */
int mm_mosaic_extract(mm_mosaic* h, const float* proj, int nth, float* const* dir, float* const* mir,
                      void* stream);
/* Replaces the blend loop of step6_stitch.py:206-262 for nth output angles:
 *   dir[p] / mir[p] point at (nth, h_p, w_p) frames of tile p's direct angles
 *   and its mirror angles (tile[t] and tile[t + N_HALF]); out (nth, nz, n)
 *   float32 receives sum(w * direct + w * flip(mirror)) / sum(w), or 1.0
 *   where no footprint covers the pixel, bit-identical to the reference's
 *   float32 arithmetic. */
int mm_mosaic_stitch(mm_mosaic* h, float* const* dir, float* const* mir, int nth, float* out, void* stream);
/* Coverage cells along rows and columns and the most footprints over one pixel. */
int mm_mosaic_info(const mm_mosaic* h, int* cells_r, int* cells_c, int* max_cover);
size_t mm_mosaic_workspace_bytes(const mm_mosaic* h);

#ifdef __cplusplus
}
#endif
#endif
