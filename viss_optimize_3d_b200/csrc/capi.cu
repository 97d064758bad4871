// capi.cu -- the extern "C" boundary (include/viss.h) and the plan.
//
// The reference reports failures through CHECK (error.cuh:4-19), which prints
// and calls exit(1).  Every entry point here returns a status instead and
// records the message in a thread-local string (viss_last_error).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "viss.h"
#include "viss_common.cuh"

namespace viss {
// launchers (healpix.cu, geometry.cu, visibility.cu, dcf.cu)
cudaError_t launch_mk_pix2xy(int32_t *, int32_t *, cudaStream_t);
cudaError_t launch_pix2ang(long long, int, long long, long long, double *, double *, double *, int,
                           cudaStream_t);
cudaError_t launch_pix_convert(long long, int, int, long long *, cudaStream_t);
cudaError_t launch_sky_pre(long long, const float *, const float *, const float *, float, double *,
                           float *, cudaStream_t);
cudaError_t launch_occulters(long long, const double *, double, int, double, double4 *,
                             cudaStream_t);
cudaError_t launch_mask_bits(long long, long long, const double *, const int32_t *,
                             const double4 *, uint32_t *, cudaStream_t);
cudaError_t launch_pix_keys(long long, const double *, unsigned long long *, int *, cudaStream_t);
cudaError_t sort_pixel_keys(long long, unsigned long long *, unsigned long long *, int *, int *,
                            cudaStream_t);
cudaError_t launch_stage_pixels(long long, long long, const double *, const int *, double4 *,
                                float4 *, cudaStream_t);
cudaError_t launch_occ32(long long, const double4 *, float4 *, cudaStream_t);
cudaError_t launch_form_stage(long long, int, const double *, const double *, double4 *,
                              unsigned long long *, cudaStream_t);
cudaError_t launch_form_stage_coef(long long, int, const float2 *, const double *, float2 *,
                                   cudaStream_t);
cudaError_t launch_form_reduce_fwd(long long, int, const double2 *, const double *, float2 *, int,
                                   cudaStream_t);
cudaError_t launch_stage_sky(long long, long long, const double4 *, const int *, const float *,
                             float, double4 *, int, cudaStream_t);
cudaError_t launch_stage_coef(long long, long long, const float2 *, float2 *, cudaStream_t);
cudaError_t launch_stage_samples(long long, const double *, const double *, const int32_t *,
                                 long long, double4 *, int4 *, unsigned long long *, int *,
                                 cudaStream_t);
cudaError_t launch_dcf(long long, const float *, int, int, int32_t *, unsigned int *, float *,
                       int, cudaStream_t);
cudaError_t launch_weights(long long, const float *, const float *, const int32_t *,
                           const float *, int, float *, float *, cudaStream_t);
cudaError_t launch_wrot(long long, const float *, float2 *, cudaStream_t);
cudaError_t launch_conj_mirror(long long, float2 *, cudaStream_t);
cudaError_t launch_scale_coef(long long, const float *, const float2 *, float2 *, cudaStream_t);
int gridded_adjoint(void **state, long long J, const double4 *pix, const int *perm, long long K,
                    const double4 *samp, const float2 *coef, int use_off, long long facet_pix, float scale,
                    float *img, int accumulate, long long max_cells, cudaStream_t st, int *grid_dims,
                    long long *facet_used, long long *info, const int4 *refs, const float4 *occ32,
                    const float4 **fcones_out, const unsigned **mixbits_out, long long *mix_words_out,
                    long long geom_version);
void gridded_free(void *state);
}  // namespace viss

#include "visibility.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int status, const std::string &msg) {
  g_last_error = msg;
  return status;
}

}  // namespace

namespace viss {
// Lets other translation units of the library record a failure message.
int record_error(int status, const std::string &msg) { return fail(status, msg); }

// Test hook of viss_forward_noalloc (armed by viss_plan_debug_drop_copy with
// a NULL plan): the tile the next call's first block skips, -1 for none;
// taking it disarms it.
namespace {
std::atomic<int> g_noalloc_drop_tile{-1};
}
int take_noalloc_drop_tile() { return g_noalloc_drop_tile.exchange(-1); }
}  // namespace viss

namespace {

int cuda_fail(cudaError_t e, const char *where) {
  g_last_error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return VISS_ERR_CUDA;
}

#define VISS_CUDA(call, where)                       \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, where); \
  } while (0)

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
  return n > 0 ? n : 148;
}

template <class T>
int ensure(T *&ptr, size_t &cap, size_t bytes, const char *what) {
  if (bytes <= cap && ptr) return VISS_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(VISS_ERR_ALLOC, std::string("cudaMalloc failed for ") + what + " (" +
                                    std::to_string(bytes) + " bytes)");
  }
  ptr = static_cast<T *>(p);
  cap = bytes;
  return VISS_OK;
}

}  // namespace

struct viss_plan {
  int device = 0;
  int nsm = 148;
  // pixels
  long long J = 0, Jpad = 0;
  int ntiles = 0;
  double4 *pix = nullptr;    size_t pix_cap = 0;
  double4 *pixsky = nullptr; size_t pixsky_cap = 0;
  float4 *cones = nullptr;   size_t cones_cap = 0;  // tile cones, then sub-tile cones
  int *perm = nullptr;       size_t perm_cap = 0;  // record i holds caller pixel perm[i]
  // samples
  long long K = 0, Kpad = 0;
  int channels = 1;        // channel-major sample axis: K = channels * Kc
  long long Kc = 0;
  double4 *samp = nullptr; size_t samp_cap = 0;
  int4 *refs = nullptr;    size_t refs_cap = 0;
  bool has_refs = false;
  double4 *occ = nullptr;  size_t occ_cap = 0;
  float4 *occ32 = nullptr; size_t occ32_cap = 0;  // classification rows
  long long G = 0;
  float2 *coef = nullptr;  size_t coef_cap = 0;
  double max_turns = 0;
  // satellite-formation mode (viss_plan_set_formation)
  long long form_T = 0;         // snapshots, all channels
  int form_S = 0;
  int form_C = 1;               // channels (viss_plan_set_formation_channels)
  double4 *form_U = nullptr;    size_t form_U_cap = 0;
  double *form_off = nullptr;   size_t form_off_cap = 0;
  bool form_has_off = false;
  double4 *form_occ = nullptr;  size_t form_occ_cap = 0;   // [T*S satellites][T snapshots]
  float4 *form_occ32 = nullptr; size_t form_occ32_cap = 0;
  int form_sat = 0, form_snap = 0;
  float2 *form_coef = nullptr;  size_t form_coef_cap = 0;
  // workspace + device status words
  void *part = nullptr;    size_t part_cap = 0;
  // [0] terms evaluated, [1] error flags, [2] terms evaluated in mixed tiles,
  // [3] |u|+|v|+|w|+|off| bound of the staged samples
  unsigned long long *dev_words = nullptr;
  size_t dev_words_cap = 0;
  long long last_total = 0;
  cudaStream_t last_stream = nullptr;
  // launch shape
  int fwd_shape = 0;   // index into viss::kFwdShapes (viss_plan_tune picks it)
  int adj_shape = 0;   // index into viss::kAdjShapes
  int drop_tile = -1;  // test hook for the next kernel (viss_plan_debug_drop_copy)
  int fwd_waves = 16;
  int adj_waves = 16;
  // viss_adjoint_gridded: its buffers and FFT plan, and what the last call used
  void *gridded = nullptr;
  int gridded_dims[3] = {0, 0, 0};
  long long gridded_facet = 0;
  long long gridded_hbm_blocks = 0;
  long long geom_version = 0;   // bumped by every call that restages pixels or samples
};

namespace {

int fwd_chunks(const viss_plan *p, int shape, bool fp64) {
  const long long per = viss::forward_samples_per_block(shape, fp64);
  const long long blocks = (p->Kc + per - 1) / per * p->channels;
  const long long slots = static_cast<long long>(p->nsm) * viss::forward_ctas_per_sm(shape, fp64);
  long long c = (static_cast<long long>(p->fwd_waves) * slots + blocks - 1) / blocks;
  c = std::max<long long>(1, std::min<long long>(c, std::max(1, p->ntiles / 2)));
  return static_cast<int>(c);
}

// Sample chunks per channel for the adjoint (and their size, a multiple of
// the staging tile).
int adj_chunks(const viss_plan *p, int shape, bool fp64, int *samples_per_chunk) {
  const long long per = viss::adjoint_pixels_per_block(shape, fp64);  // pixels per CTA
  const long long blocks = (p->Jpad + per - 1) / per * p->channels;
  const long long slots = static_cast<long long>(p->nsm) * viss::adjoint_ctas_per_sm(shape, fp64);
  long long c = (static_cast<long long>(p->adj_waves) * slots + blocks - 1) / blocks;
  const long long max_c = std::max<long long>(1, (p->Kc + 255) / 256);
  c = std::max<long long>(1, std::min(c, max_c));
  c = std::min<long long>(c, std::max<long long>(1, 65535 / p->channels));
  long long spc = (p->Kc + c - 1) / c;
  spc = (spc + viss::kSampTile - 1) / viss::kSampTile * viss::kSampTile;
  c = (p->Kc + spc - 1) / spc;
  *samples_per_chunk = static_cast<int>(spc);
  return static_cast<int>(std::max<long long>(1, c));
}

cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

int viss_version(void) { return 1; }

const char *viss_status_string(int status) {
  switch (status) {
    case VISS_OK: return "ok";
    case VISS_ERR_ARG: return "invalid argument";
    case VISS_ERR_CUDA: return "CUDA runtime error";
    case VISS_ERR_ALLOC: return "device allocation failed";
    case VISS_ERR_TIMEOUT: return "bounded device wait gave up";
    case VISS_ERR_NOTFINITE: return "non-finite input";
    case VISS_ERR_IO: return "file missing or malformed";
    case VISS_ERR_STATE: return "plan state incomplete";
    default: return "unknown status";
  }
}

size_t viss_last_error(char *buf, size_t len) {
  if (buf && len) {
    const size_t n = std::min(len - 1, g_last_error.size());
    std::memcpy(buf, g_last_error.data(), n);
    buf[n] = '\0';
  }
  return g_last_error.size();
}

// ----------------------------------------------------------------- HEALPix
int viss_mk_pix2xy(int32_t *pix2x, int32_t *pix2y, void *stream) {
  if (!pix2x || !pix2y) return fail(VISS_ERR_ARG, "viss_mk_pix2xy: null output");
  VISS_CUDA(viss::launch_mk_pix2xy(pix2x, pix2y, as_stream(stream)), "viss_mk_pix2xy");
  return VISS_OK;
}

static int check_nside(int nside, const char *who) {
  if (nside < 1 || nside > (1 << 13))
    return fail(VISS_ERR_ARG, std::string(who) + ": nside must be in [1, 8192]");
  return VISS_OK;
}

int viss_pix2ang(int nside, int scheme, int64_t first, int64_t count, double *theta, double *phi,
                 double *xyz, void *stream) {
  if (int s = check_nside(nside, "viss_pix2ang")) return s;
  const long long npix = 12LL * nside * nside;
  if (scheme != VISS_RING && scheme != VISS_NESTED)
    return fail(VISS_ERR_ARG, "viss_pix2ang: scheme must be VISS_RING or VISS_NESTED");
  if (first < 0 || count < 0 || first + count > npix)
    return fail(VISS_ERR_ARG, "viss_pix2ang: pixel range outside [0, 12 nside^2)");
  VISS_CUDA(viss::launch_pix2ang(nside, scheme, first, count, theta, phi, xyz, 0, as_stream(stream)),
            "viss_pix2ang");
  return VISS_OK;
}

int viss_pix_convert(int nside, int from_scheme, int to_scheme, int64_t *out, void *stream) {
  if (int s = check_nside(nside, "viss_pix_convert")) return s;
  if (!out) return fail(VISS_ERR_ARG, "viss_pix_convert: null output");
  if ((from_scheme != 0 && from_scheme != 1) || (to_scheme != 0 && to_scheme != 1))
    return fail(VISS_ERR_ARG, "viss_pix_convert: bad scheme");
  VISS_CUDA(viss::launch_pix_convert(nside, from_scheme, to_scheme,
                                     reinterpret_cast<long long *>(out), as_stream(stream)),
            "viss_pix_convert");
  return VISS_OK;
}

int viss_pix2lmn(int nside, int scheme, double *lmn, void *stream) {
  if (int s = check_nside(nside, "viss_pix2lmn")) return s;
  if (!lmn) return fail(VISS_ERR_ARG, "viss_pix2lmn: null output");
  if (scheme != VISS_RING && scheme != VISS_NESTED) return fail(VISS_ERR_ARG, "viss_pix2lmn: bad scheme");
  const long long npix = 12LL * nside * nside;
  VISS_CUDA(viss::launch_pix2ang(nside, scheme, 0, npix, nullptr, nullptr, lmn, 1, as_stream(stream)),
            "viss_pix2lmn");
  return VISS_OK;
}

int viss_sky_pre(int64_t npix, const float *theta, const float *phi, const float *B, float s,
                 double *lmn, float *B_out, void *stream) {
  if (npix < 0 || !theta || !phi || !lmn || (B_out && !B))
    return fail(VISS_ERR_ARG, "viss_sky_pre: bad arguments");
  VISS_CUDA(viss::launch_sky_pre(npix, theta, phi, B, s, lmn, B_out, as_stream(stream)),
            "viss_sky_pre");
  return VISS_OK;
}

// --------------------------------------------------------------- occulters
double viss_cone_threshold(float R, float h) {
  // vissgen3d_blockage.cu:251-252, on the host in FP32 like the reference.
  const float th = asinf(R / (R + h));
  const float ph = static_cast<float>(M_PI - static_cast<double>(th));
  return std::cos(static_cast<double>(ph));
}

int viss_occulters(int64_t n, const double *P, double R, int mode, double fixed_thr, double *occ,
                   void *stream) {
  if (n < 0 || (n > 0 && (!P || !occ)) || (mode != 0 && mode != 1))
    return fail(VISS_ERR_ARG, "viss_occulters: bad arguments");
  if (mode == 0 && !(R > 0)) return fail(VISS_ERR_ARG, "viss_occulters: R must be > 0");
  if (reinterpret_cast<uintptr_t>(occ) % 16)
    return fail(VISS_ERR_ARG, "viss_occulters: occ must be 16-byte aligned");
  VISS_CUDA(viss::launch_occulters(n, P, R, mode, fixed_thr, reinterpret_cast<double4 *>(occ),
                                   as_stream(stream)),
            "viss_occulters");
  return VISS_OK;
}

int viss_mask_bits(int64_t K, int64_t J, const double *lmn, const int32_t *refs, const double *occ,
                   uint32_t *bits, void *stream) {
  if (K < 0 || J < 0 || (K > 0 && J > 0 && (!lmn || !refs || !occ || !bits)))
    return fail(VISS_ERR_ARG, "viss_mask_bits: bad arguments");
  if (reinterpret_cast<uintptr_t>(occ) % 16)
    return fail(VISS_ERR_ARG, "viss_mask_bits: occ must be 16-byte aligned");
  VISS_CUDA(viss::launch_mask_bits(K, J, lmn, refs, reinterpret_cast<const double4 *>(occ), bits,
                                   as_stream(stream)),
            "viss_mask_bits");
  return VISS_OK;
}

// ------------------------------------------------------------------- plans
int viss_plan_create(viss_plan **plan) {
  if (!plan) return fail(VISS_ERR_ARG, "viss_plan_create: null plan");
  viss_plan *p = new (std::nothrow) viss_plan();
  if (!p) return fail(VISS_ERR_ALLOC, "viss_plan_create: out of host memory");
  VISS_CUDA(cudaGetDevice(&p->device), "viss_plan_create");
  p->nsm = sm_count();
  if (int s = ensure(p->dev_words, p->dev_words_cap, 4 * sizeof(unsigned long long), "status words")) {
    delete p;
    return s;
  }
  cudaMemset(p->dev_words, 0, 4 * sizeof(unsigned long long));
  *plan = p;
  return VISS_OK;
}

int viss_plan_destroy(viss_plan *p) {
  if (!p) return VISS_OK;
  void *bufs[] = {p->pix,    p->pixsky,  p->cones,    p->perm,      p->samp,
                  p->refs,   p->occ,     p->occ32,    p->coef,      p->part,
                  p->dev_words, p->form_U, p->form_off, p->form_occ, p->form_occ32,
                  p->form_coef};
  for (void *b : bufs)
    if (b) cudaFree(b);
  if (p->gridded) viss::gridded_free(p->gridded);
  delete p;
  return VISS_OK;
}

int viss_plan_set_pixels(viss_plan *p, int64_t J, const double *lmn, void *stream) {
  if (p) ++p->geom_version;
  if (!p || J <= 0 || !lmn) return fail(VISS_ERR_ARG, "viss_plan_set_pixels: bad arguments");
  if (J > (1LL << 31) * viss::kTilePix / 2)
    return fail(VISS_ERR_ARG, "viss_plan_set_pixels: too many pixels");
  // whole warp tiles of the adjoint (2 cone tiles = 256 pixels)
  const long long Jpad = (J + 2 * viss::kTilePix - 1) / (2 * viss::kTilePix) * (2 * viss::kTilePix);
  const long long nt = Jpad / viss::kTilePix;
  if (int s = ensure(p->pix, p->pix_cap, sizeof(double4) * Jpad, "pixel records")) return s;
  if (int s = ensure(p->pixsky, p->pixsky_cap, sizeof(double4) * Jpad, "pixel+sky records")) return s;
  if (int s = ensure(p->cones, p->cones_cap, sizeof(float4) * viss::cone_count(nt), "tile cones"))
    return s;
  if (int s = ensure(p->perm, p->perm_cap, sizeof(int) * J, "pixel order")) return s;
  const cudaStream_t st = as_stream(stream);
  // compact tiles: order the pixels by a hierarchical (NESTED) locality key
  void *tmp = nullptr;
  const size_t kbytes = sizeof(unsigned long long) * J, ibytes = sizeof(int) * J;
  VISS_CUDA(cudaMallocAsync(&tmp, 2 * kbytes + ibytes, st), "viss_plan_set_pixels: keys");
  auto *keys = static_cast<unsigned long long *>(tmp);
  auto *idx = reinterpret_cast<int *>(keys + 2 * J);
  cudaError_t e = viss::launch_pix_keys(J, lmn, keys, idx, st);
  if (e == cudaSuccess) e = viss::sort_pixel_keys(J, keys, keys + J, idx, p->perm, st);
  cudaError_t e2 = cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) return cuda_fail(e, "viss_plan_set_pixels: order");
  if (e2 != cudaSuccess) return cuda_fail(e2, "viss_plan_set_pixels: free");
  VISS_CUDA(viss::launch_stage_pixels(J, Jpad, lmn, p->perm, p->pix, p->cones, st),
            "viss_plan_set_pixels");
  p->J = J;
  p->Jpad = Jpad;
  p->ntiles = static_cast<int>(nt);
  return VISS_OK;
}

int viss_plan_set_samples(viss_plan *p, int64_t K, const double *uvw, const double *off,
                          const int32_t *refs, int64_t G, const double *occ, void *stream) {
  if (p) ++p->geom_version;
  if (!p || K <= 0 || !uvw) return fail(VISS_ERR_ARG, "viss_plan_set_samples: bad arguments");
  if (refs && (G <= 0 || !occ))
    return fail(VISS_ERR_ARG, "viss_plan_set_samples: refs given without an occulter table");
  if (K > (1LL << 40)) return fail(VISS_ERR_ARG, "viss_plan_set_samples: too many samples");
  const cudaStream_t st = as_stream(stream);
  const long long Kpad = (K + 1) & ~1LL;
  if (int s = ensure(p->samp, p->samp_cap, sizeof(double4) * Kpad, "sample records")) return s;
  if (int s = ensure(p->coef, p->coef_cap, sizeof(float2) * Kpad, "coefficients")) return s;
  if (refs) {
    if (int s = ensure(p->refs, p->refs_cap, sizeof(int4) * Kpad, "occulter refs")) return s;
    if (int s = ensure(p->occ, p->occ_cap, sizeof(double4) * G, "occulter table")) return s;
    if (int s = ensure(p->occ32, p->occ32_cap, sizeof(float4) * G, "occulter table")) return s;
    VISS_CUDA(cudaMemcpyAsync(p->occ, occ, sizeof(double4) * G, cudaMemcpyDeviceToDevice, st),
              "viss_plan_set_samples: occulters");
    VISS_CUDA(viss::launch_occ32(G, p->occ, p->occ32, st), "viss_plan_set_samples: occulters");
  }
  // words [1] (bad-ref flag here; error flags during a kernel) and [3] (phase bound)
  VISS_CUDA(cudaMemsetAsync(p->dev_words + 1, 0, 3 * sizeof(unsigned long long), st),
            "viss_plan_set_samples");
  p->K = 0;  // not usable until staged and checked
  VISS_CUDA(viss::launch_stage_samples(K, uvw, off, refs, refs ? G : 0, p->samp,
                                       refs ? p->refs : nullptr, p->dev_words + 3,
                                       reinterpret_cast<int *>(p->dev_words + 1), st),
            "viss_plan_set_samples");
  unsigned long long words[3] = {0, 0, 0};
  VISS_CUDA(cudaMemcpyAsync(words, p->dev_words + 1, sizeof(words), cudaMemcpyDeviceToHost, st),
            "viss_plan_set_samples: bound");
  VISS_CUDA(cudaStreamSynchronize(st), "viss_plan_set_samples: sync");
  if (static_cast<int>(words[0] & 0xffffffffu) != 0)
    return fail(VISS_ERR_ARG, "viss_plan_set_samples: occulter refs outside [-1, G)");
  double bound;
  std::memcpy(&bound, &words[2], sizeof(bound));
  if (!std::isfinite(bound))
    return fail(VISS_ERR_NOTFINITE, "viss_plan_set_samples: non-finite uvw or offset");
  p->K = K;
  p->Kpad = Kpad;
  p->channels = 1;
  p->Kc = K;
  p->has_refs = refs != nullptr;
  p->G = refs ? G : 0;
  p->max_turns = bound;
  return VISS_OK;
}

static int workspace(viss_plan *p, size_t bytes) {
  return ensure(p->part, p->part_cap, bytes, "partial-sum workspace");
}

static int forward_impl(viss_plan *p, const float *sky, float *V, int flags, cudaStream_t st,
                        int shape) {
  const bool fp64 = (flags & VISS_FP64) != 0;
  const bool masked = p->has_refs && !(flags & VISS_NO_MASK);
  const int nchunk = fwd_chunks(p, shape, fp64);
  if (int s = workspace(p, sizeof(double2) * static_cast<size_t>(nchunk) * p->K)) return s;
  if (int s = ensure(p->pixsky, p->pixsky_cap, sizeof(double4) * p->Jpad * p->channels,
                     "pixel+sky records"))
    return s;
  VISS_CUDA(viss::launch_stage_sky(p->J, p->Jpad, p->pix, p->perm, sky, 1.0f, p->pixsky,
                                   p->channels, st),
            "viss_forward: sky");
  VISS_CUDA(cudaMemsetAsync(p->dev_words, 0, 3 * sizeof(unsigned long long), st), "viss_forward");
  viss::FwdParams fp;
  fp.samp = p->samp;
  fp.refs = masked ? p->refs : nullptr;
  fp.occ = masked ? p->occ : nullptr;
  fp.occ32 = masked ? p->occ32 : nullptr;
  fp.pix = p->pixsky;
  fp.cones = p->cones;
  fp.K = p->K;
  fp.ntiles = p->ntiles;
  fp.tiles_per_chunk = (p->ntiles + nchunk - 1) / nchunk;
  const int real_chunks = (p->ntiles + fp.tiles_per_chunk - 1) / fp.tiles_per_chunk;
  fp.part = static_cast<double2 *>(p->part);
  fp.counter = p->dev_words;
  fp.err = reinterpret_cast<int *>(p->dev_words + 1);
  fp.use_off = (flags & VISS_NO_OFFSET) ? 0 : 1;
  fp.channels = p->channels;
  fp.Kc = p->Kc;
  fp.pix_stride = p->Jpad;
  fp.drop_tile = p->drop_tile;
  p->drop_tile = -1;
  VISS_CUDA(viss::launch_forward(fp, shape, real_chunks, masked, fp64, st), "viss_forward: kernel");
  VISS_CUDA(viss::launch_reduce_fwd(p->K, real_chunks, fp.part, reinterpret_cast<float2 *>(V),
                                    (flags & VISS_ACCUMULATE) ? 1 : 0, st),
            "viss_forward: reduce");
  p->last_total = p->K * p->J;
  p->last_stream = st;
  return VISS_OK;
}

static int check_call(viss_plan *p, const void *in, const void *out, int flags, const char *who) {
  if (!p || !in || !out) return fail(VISS_ERR_ARG, std::string(who) + ": bad arguments");
  if (p->J <= 0 || p->K <= 0)
    return fail(VISS_ERR_STATE, std::string(who) + ": pixels or samples not set");
  if (!(flags & VISS_FP64) && !(p->max_turns < viss::kMaxTurns))
    return fail(VISS_ERR_ARG, std::string(who) + ": |u|+|v|+|w|+|off| exceeds 2^28 turns; use VISS_FP64");
  return VISS_OK;
}

// One NVTX range per forward / adjoint call (host side; visible to profilers).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

int viss_forward(viss_plan *p, const float *sky, float *V, int flags, void *stream) {
  const NvtxRange range("viss_forward");
  if (int s = check_call(p, sky, V, flags, "viss_forward")) return s;
  return forward_impl(p, sky, V, flags, as_stream(stream), p->fwd_shape);
}

// fcones non-null: the hybrid instance (occulted, split precision), which
// leaves the (sample, facet) pairs of wholly visible facets to the gridded
// adjoint; facets of facet_pix records, nfacets of them.
static int adjoint_impl(viss_plan *p, const float *coef, float *image, float scale, int flags,
                        cudaStream_t st, int shape, const float4 *fcones = nullptr, long long facet_pix = 0,
                        long long nfacets = 0, const unsigned *mixbits = nullptr, long long mix_words = 0) {
  const bool fp64 = (flags & VISS_FP64) != 0;
  const bool masked = p->has_refs && !(flags & VISS_NO_MASK);
  int spc = 0;
  const int nchunk = adj_chunks(p, shape, fp64, &spc);
  if (int s = workspace(p, sizeof(double) * static_cast<size_t>(nchunk) * p->channels * p->Jpad))
    return s;
  VISS_CUDA(viss::launch_stage_coef(p->K, p->Kpad, reinterpret_cast<const float2 *>(coef), p->coef, st),
            "viss_adjoint: coef");
  VISS_CUDA(cudaMemsetAsync(p->dev_words, 0, 3 * sizeof(unsigned long long), st), "viss_adjoint");
  viss::AdjParams ap;
  ap.samp = p->samp;
  ap.coef = p->coef;
  ap.refs = masked ? p->refs : nullptr;
  ap.occ = masked ? p->occ : nullptr;
  ap.occ32 = masked ? p->occ32 : nullptr;
  ap.pix = p->pix;
  ap.cones = p->cones;
  ap.K = p->K;
  ap.Jpad = p->Jpad;
  ap.samples_per_chunk = spc;
  ap.part = static_cast<double *>(p->part);
  ap.counter = p->dev_words;
  ap.err = reinterpret_cast<int *>(p->dev_words + 1);
  ap.use_off = (flags & VISS_NO_OFFSET) ? 0 : 1;
  ap.channels = p->channels;
  ap.Kc = p->Kc;
  ap.nchunk = nchunk;
  ap.drop_tile = p->drop_tile;
  p->drop_tile = -1;
  if (fcones) {
    if (!masked || fp64) return fail(VISS_ERR_ARG, "viss_adjoint: the hybrid adjoint is occulted split precision");
    ap.fcones = fcones;
    ap.facet_pix = facet_pix;
    ap.nfacets = nfacets;
    ap.mixbits = mixbits;
    ap.mix_words = mix_words;
    VISS_CUDA(viss::launch_adjoint_hybrid(ap, shape, nchunk, st), "viss_adjoint_gridded: direct kernel");
  } else {
    VISS_CUDA(viss::launch_adjoint(ap, shape, nchunk, masked, fp64, st), "viss_adjoint: kernel");
  }
  VISS_CUDA(viss::launch_reduce_adj(p->J, p->Jpad, nchunk, p->channels, ap.part, p->perm, scale, image,
                                    (flags & VISS_ACCUMULATE) ? 1 : 0, st),
            "viss_adjoint: reduce");
  p->last_total = p->K * p->J;
  p->last_stream = st;
  return VISS_OK;
}

int viss_adjoint(viss_plan *p, const float *coef, float *image, float scale, int flags, void *stream) {
  const NvtxRange range("viss_adjoint");
  if (int s = check_call(p, coef, image, flags, "viss_adjoint")) return s;
  return adjoint_impl(p, coef, image, scale, flags, as_stream(stream), p->adj_shape);
}

// Times every launch shape of both kernels on this plan's problem (one warm-up
// and one timed launch each, CUDA events on `stream`) and keeps the fastest.
// Synchronous; call before capturing the plan's calls in a CUDA graph.
int viss_plan_tune(viss_plan *p, const float *sky, const float *coef, float *V_scratch,
                   float *img_scratch, int flags, int *fwd_shape, int *adj_shape, void *stream) {
  if (int s = check_call(p, sky, V_scratch, flags, "viss_plan_tune")) return s;
  if (!coef || !img_scratch) return fail(VISS_ERR_ARG, "viss_plan_tune: bad arguments");
  if (flags & VISS_FP64) return fail(VISS_ERR_ARG, "viss_plan_tune: tunes the split path only");
  const cudaStream_t st = as_stream(stream);
  cudaEvent_t e0, e1;
  VISS_CUDA(cudaEventCreate(&e0), "viss_plan_tune");
  VISS_CUDA(cudaEventCreate(&e1), "viss_plan_tune");
  float best_f = 1e30f, best_a = 1e30f;
  int bf = p->fwd_shape, ba = p->adj_shape, status = VISS_OK;
  for (int s = 0; s < viss::kNumFwdShapes && status == VISS_OK; ++s) {
    status = forward_impl(p, sky, V_scratch, flags, st, s);
    if (status) break;
    cudaEventRecord(e0, st);
    status = forward_impl(p, sky, V_scratch, flags, st, s);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) { status = cuda_fail(cudaGetLastError(), "viss_plan_tune"); break; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_f) { best_f = ms; bf = s; }
  }
  for (int s = 0; s < viss::kNumAdjShapes && status == VISS_OK; ++s) {
    status = adjoint_impl(p, coef, img_scratch, 1.0f, flags, st, s);
    if (status) break;
    cudaEventRecord(e0, st);
    status = adjoint_impl(p, coef, img_scratch, 1.0f, flags, st, s);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) { status = cuda_fail(cudaGetLastError(), "viss_plan_tune"); break; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_a) { best_a = ms; ba = s; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status) return status;
  p->fwd_shape = bf;
  p->adj_shape = ba;
  if (fwd_shape) *fwd_shape = bf;
  if (adj_shape) *adj_shape = ba;
  return VISS_OK;
}

int viss_plan_set_channels(viss_plan *p, int channels) {
  if (p) ++p->geom_version;
  if (!p || channels < 1) return fail(VISS_ERR_ARG, "viss_plan_set_channels: bad arguments");
  if (p->K <= 0) return fail(VISS_ERR_STATE, "viss_plan_set_channels: samples not set");
  if (p->K % channels != 0)
    return fail(VISS_ERR_ARG, "viss_plan_set_channels: the sample count is not a multiple of channels");
  const long long Kc = p->K / channels;
  if (channels > 1 && (Kc & 1))
    return fail(VISS_ERR_ARG, "viss_plan_set_channels: samples per channel must be even");
  if (channels > 65535) return fail(VISS_ERR_ARG, "viss_plan_set_channels: at most 65535 channels");
  p->channels = channels;
  p->Kc = Kc;
  return VISS_OK;
}

// -------------------------------------------------------- formation mode
int viss_plan_set_formation(viss_plan *p, int64_t T, int S, const double *U, const double *off,
                            const double *occ_sat, const double *occ_snap, void *stream) {
  if (!p || T < 1 || !U) return fail(VISS_ERR_ARG, "viss_plan_set_formation: bad arguments");
  if (S < 2 || S > 10)
    return fail(VISS_ERR_ARG, "viss_plan_set_formation: S must be 2 to 10 satellites");
  const long long B = viss::form_pairs(S);
  if (T * B >= (1LL << 31)) return fail(VISS_ERR_ARG, "viss_plan_set_formation: too many samples");
  const cudaStream_t st = as_stream(stream);
  const long long rows = T * S + T;
  p->form_T = 0;  // not usable until staged and checked
  if (int s = ensure(p->form_U, p->form_U_cap, sizeof(double4) * T * S, "formation vectors")) return s;
  if (int s = ensure(p->form_occ, p->form_occ_cap, sizeof(double4) * rows, "formation occulters"))
    return s;
  if (int s = ensure(p->form_occ32, p->form_occ32_cap, sizeof(float4) * rows, "formation occulters"))
    return s;
  if (off && (ensure(p->form_off, p->form_off_cap, sizeof(double) * T * B, "formation offsets")))
    return VISS_ERR_ALLOC;
  VISS_CUDA(cudaMemsetAsync(p->form_occ, 0, sizeof(double4) * rows, st), "viss_plan_set_formation");
  if (occ_sat)
    VISS_CUDA(cudaMemcpyAsync(p->form_occ, occ_sat, sizeof(double4) * T * S, cudaMemcpyDeviceToDevice, st),
              "viss_plan_set_formation: satellite rows");
  if (occ_snap)
    VISS_CUDA(cudaMemcpyAsync(p->form_occ + T * S, occ_snap, sizeof(double4) * T,
                              cudaMemcpyDeviceToDevice, st),
              "viss_plan_set_formation: snapshot rows");
  VISS_CUDA(viss::launch_occ32(rows, p->form_occ, p->form_occ32, st), "viss_plan_set_formation");
  if (off)
    VISS_CUDA(cudaMemcpyAsync(p->form_off, off, sizeof(double) * T * B, cudaMemcpyDeviceToDevice, st),
              "viss_plan_set_formation: offsets");
  VISS_CUDA(cudaMemsetAsync(p->dev_words + 3, 0, sizeof(unsigned long long), st), "viss_plan_set_formation");
  VISS_CUDA(viss::launch_form_stage(T, S, U, off, p->form_U, p->dev_words + 3, st), "viss_plan_set_formation");
  unsigned long long bits = 0;
  VISS_CUDA(cudaMemcpyAsync(&bits, p->dev_words + 3, sizeof(bits), cudaMemcpyDeviceToHost, st),
            "viss_plan_set_formation: bound");
  VISS_CUDA(cudaStreamSynchronize(st), "viss_plan_set_formation: sync");
  double bound;
  std::memcpy(&bound, &bits, sizeof(bound));
  if (!std::isfinite(bound))
    return fail(VISS_ERR_NOTFINITE, "viss_plan_set_formation: non-finite satellite vectors or offsets");
  if (!(bound < viss::kMaxTurns))
    return fail(VISS_ERR_ARG, "viss_plan_set_formation: |U| or |off| exceeds 2^28 turns");
  p->form_T = T;
  p->form_S = S;
  p->form_C = 1;
  p->form_has_off = off != nullptr;
  p->form_sat = occ_sat != nullptr;
  p->form_snap = occ_snap != nullptr;
  return VISS_OK;
}

int viss_plan_set_formation_channels(viss_plan *p, int channels) {
  if (!p || channels < 1) return fail(VISS_ERR_ARG, "viss_plan_set_formation_channels: bad arguments");
  if (p->form_T <= 0) return fail(VISS_ERR_STATE, "viss_plan_set_formation_channels: formation not set");
  if (p->form_T % channels != 0)
    return fail(VISS_ERR_ARG, "viss_plan_set_formation_channels: the snapshot count is not a multiple of channels");
  if (channels > 65535) return fail(VISS_ERR_ARG, "viss_plan_set_formation_channels: at most 65535 channels");
  p->form_C = channels;
  return VISS_OK;
}

static int check_formation(viss_plan *p, const void *in, const void *out, int flags, const char *who) {
  if (!p || !in || !out) return fail(VISS_ERR_ARG, std::string(who) + ": bad arguments");
  if (p->J <= 0 || p->form_T <= 0)
    return fail(VISS_ERR_STATE, std::string(who) + ": pixels or formation not set");
  if (flags & VISS_FP64)
    return fail(VISS_ERR_ARG, std::string(who) + ": split precision only (use viss_forward / viss_adjoint for FP64)");
  return VISS_OK;
}

static viss::FormParams form_params(viss_plan *p, int flags) {
  const bool masked = !(flags & VISS_NO_MASK);
  viss::FormParams fp{};
  fp.U = p->form_U;
  fp.occ = p->form_occ;
  fp.occ32 = p->form_occ32;
  fp.sat_rows = masked && p->form_sat;
  fp.snap_rows = masked && p->form_snap;
  fp.cones = p->cones;
  fp.ntiles = p->ntiles;
  fp.Jpad = p->Jpad;
  fp.T = p->form_T;
  fp.channels = p->form_C;
  fp.Tc = p->form_T / p->form_C;
  fp.counter = p->dev_words;
  fp.err = reinterpret_cast<int *>(p->dev_words + 1);
  return fp;
}

int viss_forward_formation(viss_plan *p, const float *sky, float *V, int flags, void *stream) {
  if (int s = check_formation(p, sky, V, flags, "viss_forward_formation")) return s;
  const NvtxRange range("viss_forward_formation");
  const cudaStream_t st = as_stream(stream);
  const long long T = p->form_T, B = viss::form_pairs(p->form_S);
  const int C = p->form_C;
  const long long Tc = T / C;
  // about 16 waves of one block per SM, each block 8 snapshots of one channel
  // x a chunk of tiles
  const long long blocks = C * ((Tc + viss::kFormFwdNT / 32 - 1) / (viss::kFormFwdNT / 32));
  long long c = (16LL * p->nsm + blocks - 1) / blocks;
  c = std::max<long long>(1, std::min<long long>(c, std::max(1, p->ntiles / 4)));
  viss::FormParams fp = form_params(p, flags);
  fp.tiles_per_chunk = static_cast<int>((p->ntiles + c - 1) / c);
  const int nchunk = (p->ntiles + fp.tiles_per_chunk - 1) / fp.tiles_per_chunk;
  fp.nchunk = nchunk;
  if (int s = workspace(p, sizeof(double2) * static_cast<size_t>(nchunk) * T * B)) return s;
  if (int s = ensure(p->pixsky, p->pixsky_cap, sizeof(double4) * p->Jpad * C, "pixel+sky records"))
    return s;
  VISS_CUDA(viss::launch_stage_sky(p->J, p->Jpad, p->pix, p->perm, sky, 1.0f, p->pixsky, C, st),
            "viss_forward_formation: sky");
  VISS_CUDA(cudaMemsetAsync(p->dev_words, 0, 3 * sizeof(unsigned long long), st), "viss_forward_formation");
  fp.pix = p->pixsky;
  fp.part_fwd = static_cast<double2 *>(p->part);
  VISS_CUDA(viss::launch_form_forward(fp, p->form_S, nchunk, st), "viss_forward_formation: kernel");
  const bool use_off = p->form_has_off && !(flags & VISS_NO_OFFSET);
  VISS_CUDA(viss::launch_form_reduce_fwd(T * B, nchunk, fp.part_fwd, use_off ? p->form_off : nullptr,
                                         reinterpret_cast<float2 *>(V), (flags & VISS_ACCUMULATE) ? 1 : 0, st),
            "viss_forward_formation: reduce");
  p->last_total = T * B * p->J;
  p->last_stream = st;
  return VISS_OK;
}

int viss_adjoint_formation(viss_plan *p, const float *coef, float *image, float scale, int flags,
                           void *stream) {
  if (int s = check_formation(p, coef, image, flags, "viss_adjoint_formation")) return s;
  const NvtxRange range("viss_adjoint_formation");
  const cudaStream_t st = as_stream(stream);
  const long long T = p->form_T, B = viss::form_pairs(p->form_S);
  const int CB = viss::form_coef_stride(p->form_S);
  if (int s = ensure(p->form_coef, p->form_coef_cap, sizeof(float2) * T * CB, "formation coefficients"))
    return s;
  const bool use_off = p->form_has_off && !(flags & VISS_NO_OFFSET);
  VISS_CUDA(viss::launch_form_stage_coef(T, p->form_S, reinterpret_cast<const float2 *>(coef),
                                         use_off ? p->form_off : nullptr, p->form_coef, st),
            "viss_adjoint_formation: coefficients");
  // chunks of each channel's snapshots: about 16 waves of CTAs in all, at
  // least 4 staging tiles per chunk
  const int C = p->form_C;
  const long long Tc = T / C;
  const long long per = viss::form_adjoint_pixels_per_block();
  const long long blocks = (p->Jpad + per - 1) / per * C;
  long long c = (16LL * p->nsm + blocks - 1) / blocks;
  const long long max_c = std::max<long long>(1, (Tc + 4 * viss::kFormSnapTile - 1) / (4 * viss::kFormSnapTile));
  c = std::max<long long>(1, std::min(c, std::min<long long>(max_c, 65535 / C)));
  long long spc = (Tc + c - 1) / c;
  spc = (spc + viss::kFormSnapTile - 1) / viss::kFormSnapTile * viss::kFormSnapTile;
  const int nchunk = static_cast<int>((Tc + spc - 1) / spc);
  if (int s = workspace(p, sizeof(double) * static_cast<size_t>(nchunk) * C * p->Jpad)) return s;
  VISS_CUDA(cudaMemsetAsync(p->dev_words, 0, 3 * sizeof(unsigned long long), st), "viss_adjoint_formation");
  viss::FormParams fp = form_params(p, flags);
  fp.pix = p->pix;
  fp.snaps_per_chunk = static_cast<int>(spc);
  fp.nchunk = nchunk;
  fp.coef = p->form_coef;
  fp.part_adj = static_cast<double *>(p->part);
  VISS_CUDA(viss::launch_form_adjoint(fp, p->form_S, nchunk, st), "viss_adjoint_formation: kernel");
  VISS_CUDA(viss::launch_reduce_adj(p->J, p->Jpad, nchunk, C, fp.part_adj, p->perm, scale, image,
                                    (flags & VISS_ACCUMULATE) ? 1 : 0, st),
            "viss_adjoint_formation: reduce");
  p->last_total = T * B * p->J;
  p->last_stream = st;
  return VISS_OK;
}

// ------------------------------------------------------ gridded adjoint
int viss_adjoint_gridded(viss_plan *p, const float *coef, float *image, float scale, int flags,
                         int64_t facet_pixels, void *stream) {
  const NvtxRange range("viss_adjoint_gridded");
  if (!p || !coef || !image) return fail(VISS_ERR_ARG, "viss_adjoint_gridded: bad arguments");
  if (p->J <= 0 || p->K <= 0) return fail(VISS_ERR_STATE, "viss_adjoint_gridded: pixels or samples not set");
  if (flags & VISS_FP64) return fail(VISS_ERR_ARG, "viss_adjoint_gridded: split precision only");
  if (p->channels != 1) return fail(VISS_ERR_ARG, "viss_adjoint_gridded: one channel only");
  if (facet_pixels < 0) return fail(VISS_ERR_ARG, "viss_adjoint_gridded: facet_pixels must be >= 0");
  const bool masked = p->has_refs && !(flags & VISS_NO_MASK);
  if (masked && !(p->max_turns < viss::kMaxTurns))
    return fail(VISS_ERR_ARG, "viss_adjoint_gridded: |u|+|v|+|w|+|off| exceeds 2^28 turns");
  const long long max_cells = 1LL << 29;   // 4 GiB of FP32 complex grid
  long long fp = facet_pixels, info = 0;
  const cudaStream_t st = as_stream(stream);
  VISS_CUDA(viss::launch_stage_coef(p->K, p->Kpad, reinterpret_cast<const float2 *>(coef), p->coef, st),
            "viss_adjoint_gridded: coef");
  const float4 *fcones = nullptr;
  const unsigned *mixbits = nullptr;
  long long mix_words = 0;
  const int s = viss::gridded_adjoint(&p->gridded, p->J, p->pix, p->perm, p->K, p->samp, p->coef,
                                      (flags & VISS_NO_OFFSET) ? 0 : 1, fp, scale, image,
                                      (flags & VISS_ACCUMULATE) ? 1 : 0, max_cells, st, p->gridded_dims, &fp,
                                      &info, masked ? p->refs : nullptr, masked ? p->occ32 : nullptr, &fcones,
                                      &mixbits, &mix_words, p->geom_version);
  p->gridded_facet = fp;
  p->gridded_hbm_blocks = info;
  p->last_stream = st;
  if (s != VISS_OK || !masked) return s;
  // the occulted adjoint: the direct kernel adds every pair the gridded part
  // left out (facets the sample does not see wholly)
  return adjoint_impl(p, coef, image, scale, (flags & ~VISS_FP64) | VISS_ACCUMULATE, st, p->adj_shape, fcones, fp,
                      (p->J + fp - 1) / fp, mixbits, mix_words);
}

int viss_plan_gridded_info(viss_plan *p, int64_t *facet_pixels, int32_t *grid_dims, int64_t *hbm_blocks) {
  if (!p) return fail(VISS_ERR_ARG, "viss_plan_gridded_info: null plan");
  if (facet_pixels) *facet_pixels = p->gridded_facet;
  if (grid_dims)
    for (int d = 0; d < 3; ++d) grid_dims[d] = p->gridded_dims[d];
  if (hbm_blocks) *hbm_blocks = p->gridded_hbm_blocks;
  return VISS_OK;
}

int viss_plan_debug_drop_copy(viss_plan *p, int tile) {
  if (tile < 0) return fail(VISS_ERR_ARG, "viss_plan_debug_drop_copy: bad arguments");
  if (!p) {
    viss::g_noalloc_drop_tile.store(tile);   // the next viss_forward_noalloc call
    return VISS_OK;
  }
  p->drop_tile = tile;
  return VISS_OK;
}

int viss_plan_set_shapes(viss_plan *p, int fwd_shape, int adj_shape) {
  if (!p || fwd_shape < 0 || fwd_shape >= viss::kNumFwdShapes || adj_shape < 0 ||
      adj_shape >= viss::kNumAdjShapes)
    return fail(VISS_ERR_ARG, "viss_plan_set_shapes: bad arguments");
  p->fwd_shape = fwd_shape;
  p->adj_shape = adj_shape;
  return VISS_OK;
}

int viss_plan_last_stats(viss_plan *p, int64_t *evaluated, int64_t *mixed, int64_t *total) {
  if (!p) return fail(VISS_ERR_ARG, "viss_plan_last_stats: null plan");
  unsigned long long w[3] = {0, 0, 0};
  VISS_CUDA(cudaStreamSynchronize(p->last_stream), "viss_plan_last_stats: sync");
  VISS_CUDA(cudaMemcpy(w, p->dev_words, sizeof(w), cudaMemcpyDeviceToHost), "viss_plan_last_stats");
  if (evaluated) *evaluated = static_cast<int64_t>(w[0]);
  if (mixed) *mixed = static_cast<int64_t>(w[2]);
  if (total) *total = p->last_total;
  if (w[1] & viss::kErrTimeout)
    return fail(VISS_ERR_TIMEOUT, "a bounded shared-memory staging wait gave up in the last kernel");
  return VISS_OK;
}

int viss_plan_last_counts(viss_plan *p, int64_t *evaluated, int64_t *total) {
  return viss_plan_last_stats(p, evaluated, nullptr, total);
}

// --------------------------------------------------------------------- DCF
int viss_dcf(int64_t n, const float *bll, int nr, int multiplicity, int32_t *gs, uint32_t *counts,
             float *dcf, void *stream) {
  if (n < 0 || nr < 1 || nr > (1 << 17) || !dcf || (n > 0 && !bll) || multiplicity < 1)
    return fail(VISS_ERR_ARG, "viss_dcf: bad arguments (nr must be in [1, 131072])");
  const cudaStream_t st = as_stream(stream);
  unsigned int *cnt = counts;
  unsigned int *tmp = nullptr;
  if (!cnt) {
    VISS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&tmp), sizeof(unsigned int) * nr, st),
              "viss_dcf: counts");
    cnt = tmp;
  }
  cudaError_t e = viss::launch_dcf(n, bll, nr, multiplicity, gs, cnt, dcf, sm_count(), st);
  if (tmp) cudaFreeAsync(tmp, st);
  if (e != cudaSuccess) return cuda_fail(e, "viss_dcf");
  return VISS_OK;
}

int viss_weights(int64_t n, const float *w, const float *bll, const int32_t *gs, const float *dcf,
                 int nr, float *dg, float *wt, void *stream) {
  if (n < 0 || (n > 0 && (!w || !bll)) || (wt && (!gs || !dcf)) || nr < 0)
    return fail(VISS_ERR_ARG, "viss_weights: bad arguments");
  VISS_CUDA(viss::launch_weights(n, w, bll, gs, dcf, nr, dg, wt, as_stream(stream)), "viss_weights");
  return VISS_OK;
}

int viss_wrot(int64_t n, const float *w, float *V, void *stream) {
  if (n < 0 || (n > 0 && (!w || !V))) return fail(VISS_ERR_ARG, "viss_wrot: bad arguments");
  VISS_CUDA(viss::launch_wrot(n, w, reinterpret_cast<float2 *>(V), as_stream(stream)), "viss_wrot");
  return VISS_OK;
}

int viss_conj_mirror(int64_t mirror, float *V, void *stream) {
  if (mirror < 0 || (mirror > 0 && !V)) return fail(VISS_ERR_ARG, "viss_conj_mirror: bad arguments");
  VISS_CUDA(viss::launch_conj_mirror(mirror, reinterpret_cast<float2 *>(V), as_stream(stream)),
            "viss_conj_mirror");
  return VISS_OK;
}

int viss_scale_coef(int64_t n, const float *wt, const float *V, float *coef, void *stream) {
  if (n < 0 || (n > 0 && (!wt || !V || !coef))) return fail(VISS_ERR_ARG, "viss_scale_coef: bad arguments");
  VISS_CUDA(viss::launch_scale_coef(n, wt, reinterpret_cast<const float2 *>(V),
                                    reinterpret_cast<float2 *>(coef), as_stream(stream)),
            "viss_scale_coef");
  return VISS_OK;
}

}  // extern "C"
