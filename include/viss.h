/*
 * viss.h -- C ABI of the B200 (sm_100a) visibility / imaging library.
 *
 * The reference (SSshuishui/viss_optimize_3d) has no library: its hot path is
 * a set of __global__ kernels driven by one host function per executable.
 * Each entry point below replaces one of those kernels or host stages; the
 * comment before it names the reference file:line it stands in for.
 *
 * Conventions
 *   - Every function returns an int status (VISS_OK == 0, negative on error)
 *     instead of the reference's CHECK -> exit(1) (error.cuh:4-19).  The text
 *     of the last failure on the calling thread is in viss_last_error().
 *   - Array arguments are DEVICE pointers owned by the caller unless the name
 *     says host_.  No function frees or keeps a caller pointer beyond the call
 *     (plans copy what they keep).
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Calls are asynchronous on that stream unless stated.
 *   - Complex arrays are interleaved (re, im) pairs.
 *   - Sky directions are the reference's (l, m, n) (vissgen3d_blockage.cu:
 *     53-74): l = sin(theta)cos(phi), m = -sin(theta)sin(phi), n = cos(theta)
 *     for a HEALPix (theta, phi).
 *   - A plan may be used from one stream at a time.
 */
#ifndef VISS_H
#define VISS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define VISS_OK 0
#define VISS_ERR_ARG (-1)       /* bad argument: NULL pointer, size out of range */
#define VISS_ERR_CUDA (-2)      /* CUDA runtime error (text in viss_last_error) */
#define VISS_ERR_ALLOC (-3)     /* device workspace allocation failed */
#define VISS_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up */
#define VISS_ERR_NOTFINITE (-5) /* NaN/inf in an input that must be finite */
#define VISS_ERR_IO (-6)        /* file missing or malformed (host drivers) */
#define VISS_ERR_STATE (-7)     /* plan used before the data it needs was set */

/* ------------------------------------------------------------------- flags */
#define VISS_FP64 0x1        /* plain FP64 path: FP64 sincos and sums */
#define VISS_NO_MASK 0x2     /* ignore occultation references */
#define VISS_NO_OFFSET 0x4   /* ignore the per-sample phase offset */
#define VISS_ACCUMULATE 0x8  /* add into the output instead of overwriting */

/* HEALPix schemes */
#define VISS_RING 0
#define VISS_NESTED 1

typedef struct viss_plan viss_plan;

int viss_version(void);
const char *viss_status_string(int status);
/* Copies the last error message of the calling thread into buf (always NUL
 * terminated when len > 0); returns the full message length. */
size_t viss_last_error(char *buf, size_t len);

/* ------------------------------------------------------------ HEALPix tables
 * Replaces pix2ang.cu:61-88 (mk_pix2xy): the 1024-entry bit de-interleave
 * tables (x = even bits, y = odd bits of a 10-bit index). Device int32[1024]. */
int viss_mk_pix2xy(int32_t *pix2x, int32_t *pix2y, void *stream);

/* Replaces pix2ang.cu:92-160 (f_pix2and_nest) and its RING twin: FP64
 * colatitude theta, longitude phi in [0, 2pi) and the HEALPix unit vector
 * (x, y, z) (count x 3) of pixels [first, first+count) in `scheme`.
 * Any of theta / phi / xyz may be NULL. */
int viss_pix2ang(int nside, int scheme, int64_t first, int64_t count, double *theta,
                 double *phi, double *xyz, void *stream);

/* Index permutation between schemes: out[p] = index in `to_scheme` of pixel p
 * of `from_scheme` (nest2ring / ring2nest), p in [0, 12 nside^2). int64. */
int viss_pix_convert(int nside, int from_scheme, int to_scheme, int64_t *out, void *stream);

/* Sky directions (l, m, n) = (x, -y, z) of the HEALPix unit vectors, FP64,
 * npix x 3 (the convention of vissgen3d_blockage.cu:53-74). */
int viss_pix2lmn(int nside, int scheme, double *lmn, void *stream);

/* ---------------------------------------------------- drop-in sky pre-pass
 * Replaces healpix_moonback_pre (vissgen3d_blockage.cu:53-74) for FP32 text
 * inputs: lmn (npix x 3, FP64) from FP32 theta/phi with the reference's angle
 * edits, and B_out = B * s.  B_out may alias B. */
int viss_sky_pre(int64_t npix, const float *theta, const float *phi, const float *B, float s,
                 double *lmn, float *B_out, void *stream);

/* ------------------------------------------------------------- occulters
 * Occulter table row (qx, qy, qz, thr): direction s is visible iff
 * fma(s2,q2, fma(s1,q1, s0*q0)) >= thr  (vissgen3d_blockage.cu:88-94).
 * From satellite positions P (n x 3, metres from the Moon's centre):
 *   mode 0: ray-sphere test against a Moon of radius R: thr = -sqrt(1-(R/|P|)^2)
 *   mode 1: the reference's fixed cone: thr = fixed_thr
 * occ is n x 4 FP64.  viss_cone_threshold gives the reference's fixed_thr
 * (vissgen3d_blockage.cu:249-252: cos(pi - asinf(R/(R+h))), host FP32 asinf). */
int viss_occulters(int64_t n, const double *P, double R, int mode, double fixed_thr,
                   double *occ, void *stream);
double viss_cone_threshold(float R, float h);

/* Mask bits for testing: bit j of row k set iff (sample k, pixel j) is
 * visible under refs (K x 3 int32 rows into occ; -1 = unused).  bits is
 * K x ceil(J/32) uint32.  Every ref must index a row of occ (the table size
 * is not passed, so this entry point cannot check it). */
int viss_mask_bits(int64_t K, int64_t J, const double *lmn, const int32_t *refs,
                   const double *occ, uint32_t *bits, void *stream);

/* ------------------------------------------------------------------ plans
 * A plan holds the pixel and sample geometry in the kernels' staging layout,
 * the tile bounding cones used to skip / fast-path occultation, the cross-
 * block partial-sum workspace and the tuned launch shapes. */
int viss_plan_create(viss_plan **plan);
int viss_plan_destroy(viss_plan *plan);

/* Pixel directions lmn (J x 3 FP64, device). */
int viss_plan_set_pixels(viss_plan *plan, int64_t J, const double *lmn, void *stream);

/* Samples: uvw (K x 3 FP64 in wavelengths), off (K FP64 turns, or NULL),
 * refs (K x 3 int32 into occ, or NULL = never occulted), occ (G x 4 FP64).
 * Refs outside [-1, G) return VISS_ERR_ARG, as do non-finite uvw or off
 * (VISS_ERR_NOTFINITE); the plan then holds no samples until the next
 * successful call.  Synchronises `stream` once. */
int viss_plan_set_samples(viss_plan *plan, int64_t K, const double *uvw, const double *off,
                          const int32_t *refs, int64_t G, const double *occ, void *stream);

/* Forward visibilities, replaces healpix_moonback_viss
 * (vissgen3d_blockage.cu:76-102):
 *   V_k = sum_j sky_j vis_kj exp(-2 pi i (u_k . s_j + off_k)),  k < K
 * sky: J FP32; V: K complex64.  Split precision by default (FP64 phase and
 * turn reduction, FP32 sincos, compensated FP32 sums, FP64 cross-block sum);
 * VISS_FP64 selects the plain FP64 path.  Asynchronous: VISS_OK means the
 * work was launched.  A bounded device-side wait that gave up inside the
 * kernel (V then incomplete) is reported only by the next
 * viss_plan_last_stats / viss_plan_last_counts on this plan, which return
 * VISS_ERR_TIMEOUT; callers that need the guarantee check it after the call. */
int viss_forward(viss_plan *plan, const float *sky, float *V, int flags, void *stream);

/* Imaging adjoint, replaces computeC (vissgen3d_blockage.cu:167-192):
 *   image_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k . s_j + off_k))) vis_kj
 * coef: K complex64 (the weighted visibilities w_k V_k); image: J FP32.
 * Asynchronous; a timed-out wait is reported as for viss_forward, only
 * through viss_plan_last_stats / viss_plan_last_counts. */
int viss_adjoint(viss_plan *plan, const float *coef, float *image, float scale, int flags,
                 void *stream);

/* Autotuner: times every launch shape of the forward and adjoint kernels on
 * this plan's problem (CUDA events on `stream`, one warm-up and one timed
 * launch each) and keeps the fastest for later calls.  sky (channels x J
 * FP32) and coef (K complex64) are representative inputs; V_scratch (K
 * complex64) and img_scratch (channels x J FP32) receive throw-away outputs.  Synchronous.  The chosen
 * shape indices are returned through fwd_shape / adj_shape (may be NULL).
 * No counterpart in the reference (it launches one fixed shape from
 * cudaOccupancyMaxPotentialBlockSize, vissgen3d_blockage.cu:412-413). */
int viss_plan_tune(viss_plan *plan, const float *sky, const float *coef, float *V_scratch,
                   float *img_scratch, int flags, int *fwd_shape, int *adj_shape, void *stream);

/* Gridded imaging adjoint: the same image as viss_adjoint (to ~1e-6
 * relative, split precision),
 *   image_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k . s_j + off_k))) vis_kj,
 * through per-facet type-3 NUFFTs.  The plan's pixel records (sorted by a
 * NESTED key) are cut into facets of `facet_pixels` records; 0 picks the size
 * 4^n with the least modelled time among those whose grid fits, from the
 * facets' measured extents.  Each facet: the samples spread onto a uniform
 * frequency grid in the facet's local frame ("exponential of semicircle"
 * kernel, width 7, oversampling 2), one FFT (cuFFT, oversampling 1.5),
 * interpolation at its pixels (width 9).
 * Unmasked (VISS_NO_MASK, or no occulter refs): computeC of the noblockage
 * programs (vissgen3d_noblockage.cu:167-182), every sample gridded.
 * Occulted: computeC of the blockage programs (vissgen3d_blockage.cu:167-192)
 * as a hybrid: a sample is gridded on the facets it sees wholly (its occulter
 * rows classify the facet's bounding cone as visible) and every other (sample,
 * facet) pair goes through the direct kernel, which skips exactly those
 * pairs; facet_pixels must then be a multiple of 256, and a timed-out wait of
 * the direct part is reported as for viss_adjoint.
 * It pays where pixels are many and baselines short against the pixel spacing
 * (Nside 512 at 1 MHz); on coarse grids or at 10 MHz viss_adjoint is faster,
 * and a sky whose grid would exceed 2^29 points for every facet size returns
 * VISS_ERR_ARG (so does an explicit facet size whose grid would).  One
 * channel; split precision only; VISS_NO_OFFSET and VISS_ACCUMULATE as for
 * viss_adjoint.  Allocates its grid (up to 2^29 complex points, 4 GiB), the
 * samples in a sorted copy and the FFT plan on first use and keeps them with
 * the plan; synchronises `stream` several times.  No counterpart in the
 * reference, whose imaging is the direct sum. */
int viss_adjoint_gridded(viss_plan *plan, const float *coef, float *image, float scale, int flags,
                         int64_t facet_pixels, void *stream);
/* What the last viss_adjoint_gridded on this plan used: facet size, grid
 * dimensions (3), and the spreading blocks whose samples did not fit one
 * shared-memory box (summed over the facets).  Any pointer may be NULL. */
int viss_plan_gridded_info(viss_plan *plan, int64_t *facet_pixels, int32_t *grid_dims, int64_t *hbm_blocks);

/* Frequency channels:the plan's K samples are `channels` consecutive blocks
 * of K/channels samples (the same baselines at each frequency; K/channels even
 * when channels > 1).  viss_forward then takes sky as channels x J (one map
 * per channel) and viss_adjoint writes image as channels x J; V and coef stay
 * K long.  All channels run in one launch of each kernel.  viss_plan_set_samples
 * resets the plan to one channel.  No counterpart in the reference (it runs one
 * frequency per executable, vissgen3d_blockage.cu:568). */
int viss_plan_set_channels(viss_plan *plan, int channels);

/* ------------------------------------------------------- formation mode
 * The samples of a satellite formation: for each of T snapshots, every pair
 * a < b of its S satellites (lexicographic order; sample k = t * S(S-1)/2 +
 * pair), with u = U[t][a] - U[t][b] (U: T x S x 3 FP64 wavelengths, e.g.
 * (P - formation centre) / lambda).  The reference builds exactly these
 * baselines (vissgen3d_blockage.cu:309-373 reads them per row); here the
 * exponential factors per satellite, e^{-2 pi i u.s} = E_a conj(E_b), so a
 * snapshot costs S exponentials per pixel instead of S(S-1)/2.  Same results
 * as viss_forward / viss_adjoint with uvw = U_a - U_b, refs = (t S + a,
 * t S + b, T S + t) and occ = [occ_sat; occ_snap] (split precision only).
 *   off      T x S(S-1)/2 phase offsets in turns, or NULL
 *   occ_sat  T x S x 4 occulter rows of the satellites (Moon), or NULL
 *   occ_snap T x 4 rows of the snapshots (Earth cap), or NULL
 * 2 <= S <= 10.  Synchronises `stream` once.  No counterpart in the
 * reference. */
int viss_plan_set_formation(viss_plan *plan, int64_t T, int S, const double *U, const double *off,
                            const double *occ_sat, const double *occ_snap, void *stream);
/* Frequency channels of a formation: the T snapshots given to
 * viss_plan_set_formation are C channels of T / C snapshots each (channel-major;
 * U scaled by each channel's wavelength, the occulter rows repeated per channel).
 * Each channel has its own sky and image; one launch per kernel covers all.
 * Reset to 1 by viss_plan_set_formation. */
int viss_plan_set_formation_channels(viss_plan *plan, int channels);
/* V (T x S(S-1)/2 complex64) for sky (C x J FP32); flags VISS_NO_MASK,
 * VISS_NO_OFFSET, VISS_ACCUMULATE (VISS_FP64 is rejected). */
int viss_forward_formation(viss_plan *plan, const float *sky, float *V, int flags, void *stream);
/* image (C x J FP32) = scale * the adjoint of the formation's samples for coef
 * (T x S(S-1)/2 complex64), each channel's samples into its own image;
 * flags VISS_NO_MASK, VISS_NO_OFFSET, VISS_ACCUMULATE (VISS_FP64 is rejected). */
int viss_adjoint_formation(viss_plan *plan, const float *coef, float *image, float scale, int flags,
                           void *stream);

/* Test hook for the failure path: the next viss_forward or viss_adjoint on
 * this plan has its first thread block skip the staging copy of its `tile`-th
 * tile (a pixel tile in the forward, a sample tile in the adjoint), so that
 * block's bounded waits give up (about 1 s each, no fault, no trap), the
 * kernel ends, and viss_plan_last_stats / viss_plan_last_counts then return
 * VISS_ERR_TIMEOUT; the plan and the context stay usable.  The results of
 * that one call are incomplete.  With plan == NULL the hook arms the next
 * viss_forward_noalloc call instead (process-wide), which then returns
 * VISS_ERR_TIMEOUT itself.  No counterpart in the reference. */
int viss_plan_debug_drop_copy(viss_plan *plan, int tile);

/* Sets the launch shapes directly (indices 0..3 each). */
int viss_plan_set_shapes(viss_plan *plan, int fwd_shape, int adj_shape);

/* Terms evaluated by the last viss_forward / viss_adjoint on this plan
 * (visible-or-mixed pairs actually exponentiated) and the total K*J, read
 * back from the device (synchronises the plan's last stream). */
int viss_plan_last_counts(viss_plan *plan, int64_t *evaluated, int64_t *total);
/* The same plus the terms evaluated in "mixed" tiles (per-term occultation
 * test).  Returns VISS_ERR_TIMEOUT if the last kernel reported a bounded
 * staging wait that gave up. */
int viss_plan_last_stats(viss_plan *plan, int64_t *evaluated, int64_t *mixed, int64_t *total);

/* Forward visibilities without any device allocation, for callers that
 * cannot call cudaMalloc (a host application that owns the device-memory
 * budget through its own pool allocator, or a pipeline that must not
 * allocate after start-up).  No counterpart in the reference.  Same result
 * as viss_forward (split precision) for lmn (J x 3), sky (J), uvw (K x 3),
 * off (K or NULL), refs (K x 3 or NULL) and occ (G x 4, 16-byte aligned);
 * V is K complex64.  All intermediates live in one fixed 9 MiB __device__
 * array that every GPU loading the library holds until the process exits.
 * Limits: J <= 65536 pixels, K <= 32768 samples, G <= 98304 occulter rows
 * (else VISS_ERR_ARG).  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress)
 * -- make it before any stream capture -- and keeps it for the life of the
 * process, so the entry point must not be used across a cudaDeviceReset.
 * Calls share the array: calls that overlap on the GPU race.  Each call
 * synchronises `stream` twice (the phase-bound check before the kernel, the
 * kernel's error word after it) and returns VISS_ERR_TIMEOUT, with V
 * incomplete, if a bounded device-side wait gave up. */
int viss_forward_noalloc(int64_t J, const double *lmn, const float *sky, int64_t K,
                         const double *uvw, const double *off, const int32_t *refs, int64_t G,
                         const double *occ, float *V, void *stream);

/* ----------------------------------------------- density compensation
 * Replaces ceilAndScale + countOccurrences + calculateR + calculateDcf
 * (vissgen3d_blockage.cu:105-141; the un-shifted formula of
 * vissgen3d_noblockage.cu:132-141):
 *   gs_i = ceil((bll_i - 1/4) / 0.5)  (FP32, as the reference)
 *   counts[p-1] = multiplicity * #{i : gs_i == p}, p in [1, nr]  (uint32)
 *   dcf[0] = 1/(4 pi); dcf[k] = (2 pi/3)(R^3 - (R-1/2)^3) / counts[k-1],
 *   R = k/2 + 1/4 (FP64, stored FP32).  gs / counts may be NULL. */
int viss_dcf(int64_t n, const float *bll, int nr, int multiplicity, int32_t *gs,
             uint32_t *counts, float *dcf, void *stream);

/* Replaces viss_gamma_trans (vissgen3d_blockage.cu:144-164), weights part:
 *   dg_i = 1.5 sqrt|1 - 4x^2| / sqrt(1 - x^2), x = w_i / bll_i (|x|>=1: inf)
 *   wt_i = min(dcf[clamp(gs_i, 0, nr)] * dg_i, 1/8)      (FP32, :178,187)
 * dg may be NULL. */
int viss_weights(int64_t n, const float *w, const float *bll, const int32_t *gs,
                 const float *dcf, int nr, float *dg, float *wt, void *stream);

/* w-rotation of viss_gamma_trans (vissgen3d_blockage.cu:150-151):
 *   V_i <- V_i exp(-2 pi i w_i)  (FP64 phase), complex64 in place; w FP32. */
int viss_wrot(int64_t n, const float *w, float *V, void *stream);

/* coef_i = wt_i * V_i (complex64), optionally conj-copied: when
 * mirror > 0, rows [mirror, 2 mirror) of V are first set to conj of rows
 * [0, mirror) (vissgen3d_blockage.cu:100). */
int viss_conj_mirror(int64_t mirror, float *V, void *stream);
int viss_scale_coef(int64_t n, const float *wt, const float *V, float *coef, void *stream);

/* ------------------------------------------------------------ day streaming
 * One observation day's rows (n = unique rows + their mirrors, as in the
 * reference's per-day files, vissgen3d_blockage.cu:309-391) staged on the
 * device: replaces the host loops of the reference's vissGen that build the
 * per-row geometry.  Inputs are FP32 rows (x, y, z) of uvw, xyza, xyzb
 * (device, n x 3 each); outputs (device): uvw (n x 3 FP64), off (n, = -w, the
 * forward's w(n-1) term, :95), P (2n x 3 FP64: satellite a of row i at row i,
 * satellite b at row n + i), refs (n x 3 int32 = (i, n + i, -1)), w (n FP32).
 * n < 2^30. */
int viss_stage_day_rows(int64_t n, const float *uvw3, const float *xyza3, const float *xyzb3,
                        double *uvw, double *off, double *P, int32_t *refs, float *w,
                        void *stream);

/* sum[j] += img[j] for n pixels in FP64, non-finite pixels counted as 0: the
 * day sum the reference's notebooks form on the host with NaN -> 0
 * (healpix3d_blockage.ipynb:103-116), kept on the device. */
int viss_accumulate_image(int64_t n, const float *img, double *sum, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* VISS_H */
