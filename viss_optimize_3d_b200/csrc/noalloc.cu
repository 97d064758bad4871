// noalloc.cu -- forward visibilities for callers that cannot allocate device
// memory.
//
// viss_forward goes through a plan, and a plan calls cudaMalloc for its
// staging buffers and cross-block workspace.  Some callers cannot do that:
// a host application that hands the library a fixed device-memory budget
// through its own pool allocator, or an observation pipeline that must not
// allocate after start-up.  viss_forward_noalloc computes the same
// visibilities with every intermediate buffer carved out of one file-scope
// __device__ array of fixed size (kScratchBytes, about 9 MiB).  That array exists
// on every GPU that loads the library, for the life of the process, whether
// or not this entry point is ever called.
//
// Limits and rules (also in include/viss.h):
//   - at most kNaMaxPix pixels, kNaMaxSamp samples and kNaMaxOcc occulter
//     rows per call; larger inputs are rejected with VISS_ERR_ARG;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current);
//     make that first call before any stream capture;
//   - all calls share the one array, so calls that overlap on the GPU (two
//     streams, two host threads) race and corrupt each other's results;
//   - each call synchronises its stream twice: once to read back the |u.s|
//     bound that decides whether the split-precision phase is valid, and once
//     at the end to read the kernel's error word, so that a bounded staging
//     wait that gave up is returned by this call as VISS_ERR_TIMEOUT;
//   - the array's address is cached per device for the life of the process;
//     after cudaDeviceReset (which unloads the module) the cached address is
//     stale, so this entry point must not be used across a device reset.
// Pixels are processed in the caller's order (no locality sort: sorting
// needs temporary storage), so tiles of a non-NESTED input are less compact
// and more of them take the per-term occultation test; results are the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "viss.h"
#include "visibility.cuh"

namespace viss {
cudaError_t launch_stage_samples(long long, const double *, const double *, const int32_t *,
                                 long long, double4 *, int4 *, unsigned long long *, int *,
                                 cudaStream_t);
cudaError_t launch_tile_cones(long long ntiles, const double4 *pix, float4 *cones,
                              cudaStream_t st);
cudaError_t launch_occ32(long long G, const double4 *occ, float4 *out, cudaStream_t st);
int record_error(int status, const std::string &msg);
int take_noalloc_drop_tile();
}  // namespace viss

namespace {

constexpr long long kNaMaxPix = 65536;   // pixels per call (Nside 64 is 49,152)
constexpr long long kNaMaxSamp = 32768;  // samples per call
constexpr long long kNaMaxOcc = 3 * kNaMaxSamp;  // occulter rows per call
constexpr int kNaMaxChunks = 8;          // cross-block partial sums per sample

// Byte offsets of the regions inside the array (each a multiple of 256).
constexpr size_t kOffPix = 0;                                        // double4[kNaMaxPix]
constexpr size_t kOffCones = kOffPix + 32ull * kNaMaxPix;            // float4[cone_count(kNaMaxPix/128)]
constexpr size_t kOffOcc32 =
    kOffCones + (16ull * viss::cone_count(kNaMaxPix / viss::kTilePix) + 255) / 256 * 256;  // float4[kNaMaxOcc]
constexpr size_t kOffSamp = kOffOcc32 + 16ull * kNaMaxOcc;           // double4[kNaMaxSamp]
constexpr size_t kOffRefs = kOffSamp + 32ull * kNaMaxSamp;           // int4[kNaMaxSamp]
constexpr size_t kOffPart = kOffRefs + 16ull * kNaMaxSamp;           // double2[chunks][kNaMaxSamp]
constexpr size_t kOffWords = kOffPart + 16ull * kNaMaxChunks * kNaMaxSamp;  // 4 x uint64
constexpr size_t kScratchBytes = kOffWords + 256;

}  // namespace

// The scratch array.  Host code must not use this name as a pointer: on the
// host it is only a handle for cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_viss_noalloc_scratch[kScratchBytes];

namespace {

// Pixel records in the caller's order: (l, m, n, sky bits), padded to Jpad
// with copies of the last pixel carrying zero sky.
__global__ void k_na_stage_pix(long long J, long long Jpad, const double *lmn, const float *sky,
                               double4 *pix) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= Jpad) return;
  const long long s = i < J ? i : J - 1;
  const float v = i < J ? sky[i] : 0.0f;
  pix[i] = make_double4(lmn[3 * s], lmn[3 * s + 1], lmn[3 * s + 2],
                        __hiloint2double(0, __float_as_int(v)));
}

std::mutex g_na_mutex;
constexpr int kNaMaxDevices = 64;
void *g_na_base[kNaMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device.
int na_scratch(unsigned char **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return viss::record_error(VISS_ERR_CUDA, std::string("viss_forward_noalloc: cudaGetDevice: ") +
                                                 cudaGetErrorString(e));
  if (dev < 0 || dev >= kNaMaxDevices)
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: device ordinal above 63");
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_base[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_viss_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return viss::record_error(VISS_ERR_CUDA,
                                std::string("viss_forward_noalloc: cudaGetSymbolAddress: ") +
                                    cudaGetErrorString(e));
    g_na_base[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_na_base[dev]);
  return VISS_OK;
}

int na_cuda(cudaError_t e, const char *where) {
  return viss::record_error(VISS_ERR_CUDA, std::string("viss_forward_noalloc: ") + where + ": " +
                                               cudaGetErrorString(e));
}

}  // namespace

extern "C" int viss_forward_noalloc(int64_t J, const double *lmn, const float *sky, int64_t K,
                                    const double *uvw, const double *off, const int32_t *refs,
                                    int64_t G, const double *occ, float *V, void *stream) {
  if (J < 1 || K < 1 || !lmn || !sky || !uvw || !V)
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: bad arguments");
  if (J > kNaMaxPix || K > kNaMaxSamp)
    return viss::record_error(
        VISS_ERR_ARG, "viss_forward_noalloc: " + std::to_string(J) + " pixels x " +
                          std::to_string(K) + " samples exceeds the fixed scratch (at most " +
                          std::to_string(kNaMaxPix) + " pixels and " + std::to_string(kNaMaxSamp) +
                          " samples); use viss_forward with a plan");
  if (refs && (G < 1 || !occ))
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: refs need an occulter table");
  if (refs && G > kNaMaxOcc)
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: " + std::to_string(G) +
                                                " occulter rows exceeds the fixed scratch (at most " +
                                                std::to_string(kNaMaxOcc) + "); use viss_forward with a plan");
  if (refs && reinterpret_cast<uintptr_t>(occ) % 16)
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: occ must be 16-byte aligned");

  unsigned char *base = nullptr;
  if (int s = na_scratch(&base)) return s;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  double4 *pix = reinterpret_cast<double4 *>(base + kOffPix);
  float4 *cones = reinterpret_cast<float4 *>(base + kOffCones);
  float4 *occ32 = reinterpret_cast<float4 *>(base + kOffOcc32);
  double4 *samp = reinterpret_cast<double4 *>(base + kOffSamp);
  int4 *ref4 = reinterpret_cast<int4 *>(base + kOffRefs);
  double2 *part = reinterpret_cast<double2 *>(base + kOffPart);
  unsigned long long *words = reinterpret_cast<unsigned long long *>(base + kOffWords);

  // whole 256-pixel units, as the plan pads them
  const long long unit = 2 * viss::kTilePix;
  const long long Jpad = (J + unit - 1) / unit * unit;
  const long long ntiles = Jpad / viss::kTilePix;

  // the previous call's words (counters, error flag, bound) must not leak in
  cudaError_t e = cudaMemsetAsync(words, 0, 4 * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return na_cuda(e, "clear");
  k_na_stage_pix<<<static_cast<unsigned>((Jpad + 255) / 256), 256, 0, st>>>(J, Jpad, lmn, sky, pix);
  if ((e = cudaGetLastError()) != cudaSuccess) return na_cuda(e, "stage pixels");
  if ((e = viss::launch_tile_cones(ntiles, pix, cones, st)) != cudaSuccess) return na_cuda(e, "cones");
  if (refs && (e = viss::launch_occ32(G, reinterpret_cast<const double4 *>(occ), occ32, st)) != cudaSuccess)
    return na_cuda(e, "occulters");
  if ((e = viss::launch_stage_samples(K, uvw, off, refs, refs ? G : 0, samp,
                                      refs ? ref4 : nullptr, words + 3,
                                      reinterpret_cast<int *>(words + 1), st)) != cudaSuccess)
    return na_cuda(e, "stage samples");

  // bad-ref flag (word 1) and the |u.s + off| bound (word 3): the split-precision
  // phase needs |u.s + off| < 2^28 turns
  unsigned long long w13[3] = {0, 0, 0};
  if ((e = cudaMemcpyAsync(w13, words + 1, sizeof(w13), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return na_cuda(e, "bound");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return na_cuda(e, "sync");
  if (static_cast<int>(w13[0] & 0xffffffffu) != 0)
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: occulter refs outside [-1, G)");
  double bound;
  std::memcpy(&bound, &w13[2], sizeof(bound));
  if (!std::isfinite(bound))
    return viss::record_error(VISS_ERR_NOTFINITE, "viss_forward_noalloc: non-finite uvw or offset");
  if (!(bound < viss::kMaxTurns))
    return viss::record_error(VISS_ERR_ARG, "viss_forward_noalloc: |u|+|v|+|w|+|off| exceeds 2^28 turns");

  // grid: about 16 waves of resident CTAs, at most kNaMaxChunks chunks
  int nsm = 148;
  int devi = 0;
  if (cudaGetDevice(&devi) == cudaSuccess)
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, devi);
  const int shape = 0;
  const long long per = viss::forward_samples_per_block(shape, false);
  const long long blocks = (K + per - 1) / per;
  const long long slots = static_cast<long long>(nsm) * viss::forward_ctas_per_sm(shape, false);
  long long nchunk = (16 * slots + blocks - 1) / blocks;
  nchunk = std::max(1LL, std::min<long long>(nchunk, std::min<long long>(kNaMaxChunks,
                                                                         std::max(1LL, ntiles / 2))));
  viss::FwdParams fp;
  fp.samp = samp;
  fp.refs = refs ? ref4 : nullptr;
  fp.occ = refs ? reinterpret_cast<const double4 *>(occ) : nullptr;
  fp.occ32 = refs ? occ32 : nullptr;
  fp.pix = pix;
  fp.cones = cones;
  fp.K = K;
  fp.ntiles = static_cast<int>(ntiles);
  fp.tiles_per_chunk = static_cast<int>((ntiles + nchunk - 1) / nchunk);
  const int real_chunks = static_cast<int>((ntiles + fp.tiles_per_chunk - 1) / fp.tiles_per_chunk);
  fp.part = part;
  fp.counter = words;
  fp.err = reinterpret_cast<int *>(words + 1);
  fp.use_off = 1;
  fp.channels = 1;
  fp.Kc = K;
  fp.pix_stride = Jpad;
  // test hook: viss_plan_debug_drop_copy(NULL, tile) arms the next call
  fp.drop_tile = viss::take_noalloc_drop_tile();
  if ((e = viss::launch_forward(fp, shape, real_chunks, refs != nullptr, false, st)) != cudaSuccess)
    return na_cuda(e, "forward kernel");
  if ((e = viss::launch_reduce_fwd(K, real_chunks, part, reinterpret_cast<float2 *>(V), 0, st)) !=
      cudaSuccess)
    return na_cuda(e, "reduce");
  // the kernel's error word: a bounded staging wait that gave up leaves V
  // incomplete, and the caller learns it here rather than never
  unsigned long long err = 0;
  if ((e = cudaMemcpyAsync(&err, words + 1, sizeof(err), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    return na_cuda(e, "error word");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return na_cuda(e, "sync");
  if (err & viss::kErrTimeout)
    return viss::record_error(VISS_ERR_TIMEOUT,
                              "viss_forward_noalloc: a bounded shared-memory staging wait gave up; "
                              "V is incomplete");
  return VISS_OK;
}
