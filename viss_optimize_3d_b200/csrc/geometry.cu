// geometry.cu -- occulter tables, mask bits, staging layouts and tile cones.
//
// The occultation predicate of the reference (vissgen3d_blockage.cu:88-94 in
// the forward kernel, :180-186 in the imaging kernel) is
//   acosf(s.P / |P|) <= phi,   phi = pi - asinf(R/(R+h))   (:249-252)
// per (sample, pixel), for both satellites of the baseline.  Here it is the
// acos-free equivalent dot(s, P/|P|) >= cos(phi), evaluated in FP64 with a
// fixed operation order (dot_exact) so that the CPU oracle reproduces every
// bit; the same form with thr = -sqrt(1 - (R/|P|)^2) is the exact ray-sphere
// test, and with q = -e, thr = -cos(rho) an Earth cap of radius rho.
#include <cub/device/device_radix_sort.cuh>

#include "viss_common.cuh"

namespace viss {

__global__ void k_occulters(long long n, const double *P, double R, int mode, double fixed_thr,
                            double4 *occ) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = P[3 * i], y = P[3 * i + 1], z = P[3 * i + 2];
  const double r = __dsqrt_rn(__fma_rn(z, z, __fma_rn(y, y, __dmul_rn(x, x))));
  double4 o;
  o.x = __ddiv_rn(x, r);
  o.y = __ddiv_rn(y, r);
  o.z = __ddiv_rn(z, r);
  if (mode == 0) {
    const double rho = __ddiv_rn(R, r);
    o.w = -__dsqrt_rn(__dadd_rn(1.0, -__dmul_rn(rho, rho)));
  } else {
    o.w = fixed_thr;
  }
  occ[i] = o;
}

__device__ __forceinline__ bool visible3(const int32_t *r, const double4 *occ, double s0,
                                         double s1, double s2) {
  for (int c = 0; c < 3; ++c) {
    const int g = r[c];
    if (g < 0) continue;
    const double4 q = occ[g];
    if (!(dot_exact(s0, s1, s2, q) >= q.w)) return false;
  }
  return true;
}

// One warp per (sample row, 32-pixel word).
__global__ void k_mask_bits(long long K, long long J, const double *lmn, const int32_t *refs,
                            const double4 *occ, uint32_t *bits) {
  const long long W = (J + 31) / 32;
  const long long word = static_cast<long long>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (word >= K * W) return;
  const long long k = word / W, jw = word - k * W;
  const long long j = jw * 32 + lane;
  bool v = false;
  if (j < J) v = visible3(refs + 3 * k, occ, lmn[3 * j], lmn[3 * j + 1], lmn[3 * j + 2]);
  const uint32_t b = __ballot_sync(0xffffffffu, v);
  if (lane == 0) bits[word] = b;
}

// Locality key of a direction: its HEALPix NESTED index at Nside 2^13
// (standard ang2pix_nest).  NESTED indices are hierarchical, so sorting by the
// key puts every 4^k-aligned run of pixels in a compact patch of sky -- for a
// HEALPix grid of any Nside <= 2^13 the sorted order is its NESTED order.
__device__ unsigned long long spread32(unsigned long long x) {
  x &= 0xffffffffull;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}

__global__ void k_pix_keys(long long J, const double *lmn, unsigned long long *keys, int *idx) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= J) return;
  const long long N = 8192;
  const double x = lmn[3 * i], y = lmn[3 * i + 1], z0 = lmn[3 * i + 2];
  const double r = sqrt(x * x + y * y + z0 * z0);
  const double z = r > 0 ? z0 / r : 1.0;
  const double za = fabs(z);
  double phi = atan2(y, x);
  if (phi < 0) phi += 2.0 * 3.141592653589793;
  double tt = phi / (0.5 * 3.141592653589793);
  if (tt >= 4.0) tt -= 4.0;
  long long face, ix, iy;
  if (za <= 2.0 / 3.0) {
    const double t1 = N * (0.5 + tt), t2 = N * z * 0.75;
    const long long jp = static_cast<long long>(t1 - t2), jm = static_cast<long long>(t1 + t2);
    const long long ifp = jp / N, ifm = jm / N;
    face = (ifp == ifm) ? (ifp | 4) : ((ifp < ifm) ? ifp : ifm + 8);
    ix = jm & (N - 1);
    iy = N - (jp & (N - 1)) - 1;
  } else {
    const long long ntt = min(3LL, static_cast<long long>(tt));
    const double tp = tt - ntt;
    const double tmp = N * sqrt(3.0 * (1.0 - za));
    const long long jp = min(N - 1, static_cast<long long>(tp * tmp));
    const long long jm = min(N - 1, static_cast<long long>((1.0 - tp) * tmp));
    if (z >= 0) { face = ntt; ix = N - jm - 1; iy = N - jp - 1; }
    else { face = ntt + 8; ix = jp; iy = jm; }
  }
  face = face < 0 ? 0 : (face > 11 ? 11 : face);
  ix = ix < 0 ? 0 : (ix >= N ? N - 1 : ix);
  iy = iy < 0 ? 0 : (iy >= N ? N - 1 : iy);
  keys[i] = static_cast<unsigned long long>(face) * N * N + spread32(ix) + (spread32(iy) << 1);
  idx[i] = static_cast<int>(i);
}

// Pixel staging: record i = pixel perm[i] of lmn (J x 3); padded to Jpad with
// copies of the last record (sky is zero there and the adjoint drops them).
__global__ void k_stage_pixels(long long J, long long Jpad, const double *lmn, const int *perm,
                               double4 *pix) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= Jpad) return;
  const long long s = perm[i < J ? i : J - 1];
  pix[i] = make_double4(lmn[3 * s], lmn[3 * s + 1], lmn[3 * s + 2], 0.0);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// FP32 centre of a pixel set with coordinate sums (sx, sy, sz): the
// normalised mean rounded to float, or (1, 0, 0) when the mean is ~0.
__device__ __forceinline__ float4 cone_centre(double sx, double sy, double sz, bool &degenerate) {
  const double nrm = sqrt(sx * sx + sy * sy + sz * sz);
  degenerate = !(nrm > 1e-6);
  if (degenerate) return make_float4(1.f, 0.f, 0.f, 0.f);
  return make_float4(__double2float_rn(sx / nrm), __double2float_rn(sy / nrm),
                     __double2float_rn(sz / nrm), 0.f);
}

__device__ __forceinline__ double chord(double x, double y, double z, const float4 &c) {
  const double dx = x - c.x, dy = y - c.y, dz = z - c.z;
  return sqrt(dx * dx + dy * dy + dz * dz);
}

// Radius field of an FP32 cone (see cone_state32): the largest chord to the
// rounded centre plus kConeMargin32, rounded up; 4 (wider than any chord of
// unit vectors) for a degenerate set, NaN if any pixel is NaN so that every
// classification falls through to the exact per-pixel test.
__device__ __forceinline__ float cone_radius(double rho, bool degenerate, bool any_nan) {
  if (any_nan) return __int_as_float(0x7fc00000);
  if (degenerate) return 4.f;
  return __double2float_ru(rho + kConeMargin32);
}

// FP32 bounding cones: cones[t] for each kTilePix-pixel tile t and
// cones[ntiles + 4 t + s] for its four 32-pixel sub-tiles (pixels
// 128 t + 32 s .. + 31).  One warp per tile; lane l holds pixels 32 s + l.
__global__ void k_tile_cones(long long ntiles, const double4 *pix, float4 *cones) {
  const long long t = static_cast<long long>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (t >= ntiles) return;
  double px[4], py[4], pz[4];
  bool nan_lane = false;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const double4 q = pix[t * kTilePix + 32 * s + lane];
    px[s] = q.x; py[s] = q.y; pz[s] = q.z;
    nan_lane = nan_lane || isnan(q.x) || isnan(q.y) || isnan(q.z);
  }
  double tx = 0, ty = 0, tz = 0;
  float4 sub[4];
  bool sub_deg[4], sub_nan[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const double sx = warp_sum(px[s]), sy = warp_sum(py[s]), sz = warp_sum(pz[s]);
    tx += sx; ty += sy; tz += sz;
    sub[s] = cone_centre(sx, sy, sz, sub_deg[s]);
    sub_nan[s] = __any_sync(0xffffffffu, isnan(px[s]) || isnan(py[s]) || isnan(pz[s]));
  }
  bool tile_deg;
  float4 tile = cone_centre(tx, ty, tz, tile_deg);
  double rho_t = 0;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const double rs = warp_max(chord(px[s], py[s], pz[s], sub[s]));
    sub[s].w = cone_radius(rs, sub_deg[s], sub_nan[s]);
    rho_t = fmax(rho_t, chord(px[s], py[s], pz[s], tile));
  }
  rho_t = warp_max(rho_t);
  tile.w = cone_radius(rho_t, tile_deg, __any_sync(0xffffffffu, nan_lane));
  if (lane < 4) cones[ntiles + 4 * t + lane] = sub[lane];
  if (lane == 0) cones[t] = tile;
}

// Super-tile cones: the cone enclosing the FP32 cones of tiles
// [kSuperTiles s, kSuperTiles (s + 1)) at cones[5 ntiles + s].  Centre =
// normalised sum of the tile centres rounded to FP32; radius = the largest
// chord to a tile centre plus that tile's radius (which already carries
// kConeMargin32), rounded up: every pixel of every tile lies within it.
__global__ void k_super_cones(long long ntiles, float4 *cones) {
  const long long s = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  const long long nsup = (ntiles + kSuperTiles - 1) / kSuperTiles;
  if (s >= nsup) return;
  const long long t0 = s * kSuperTiles, t1 = min(t0 + kSuperTiles, ntiles);
  double sx = 0, sy = 0, sz = 0;
  bool bad = false;
  for (long long t = t0; t < t1; ++t) {
    const float4 c = cones[t];
    sx += c.x; sy += c.y; sz += c.z;
    bad = bad || isnan(c.w);
  }
  bool degenerate;
  float4 sc = cone_centre(sx, sy, sz, degenerate);
  double r = 0;
  for (long long t = t0; t < t1; ++t) {
    const float4 c = cones[t];
    r = fmax(r, chord(c.x, c.y, c.z, sc) + static_cast<double>(c.w));
  }
  sc.w = bad ? __int_as_float(0x7fc00000) : (degenerate ? 4.f : __double2float_ru(r + 1e-9));
  cones[5 * ntiles + s] = sc;
}

// FP32 occulter rows for the classification: (q, thr) / |q| (the same
// half-space with a unit direction); rows with |q| = 0 or non-finite |q| are
// rounded as they are (NaN stays NaN: "test every pixel").
__global__ void k_occ32(long long G, const double4 *occ, float4 *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= G) return;
  const double4 q = occ[i];
  const double n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z);
  const double s = (n > 0.0 && n <= 1.7e308) ? 1.0 / n : 1.0;
  out[i] = make_float4(__double2float_rn(q.x * s), __double2float_rn(q.y * s),
                       __double2float_rn(q.z * s), __double2float_rn(q.w * s));
}

// Sky staging: pixel record + sky value in the low word of .w (zero past J),
// so one 32-byte record per pixel carries everything the forward reads.
// One channel per blockIdx.y: out[ch][i] = (pix[i], sky[ch][perm[i]]).
__global__ void k_stage_sky(long long J, long long Jpad, const double4 *pix, const int *perm,
                            const float *sky, float scale, double4 *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= Jpad) return;
  const long long ch = blockIdx.y;
  double4 r = pix[i];
  const float v = i < J ? __fmul_rn(sky[ch * J + perm[i]], scale) : 0.0f;
  r.w = __hiloint2double(0, __float_as_int(v));
  out[ch * Jpad + i] = r;
}

// Sample staging: uvw (K x 3), off (K or null), refs (K x 3 or null).
// Sample staging.  Occulter refs outside [-1, G) set *badref and are staged
// as -1, so the kernels never index past the occulter table.
__device__ __forceinline__ int checked_ref(int r, long long G, int *badref) {
  if (r < -1 || r >= G) {
    atomicOr(badref, 1);
    return -1;
  }
  return r;
}

__global__ void k_stage_samples(long long K, const double *uvw, const double *off,
                                const int32_t *refs, long long G, double4 *samp, int4 *ref4,
                                int *badref) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K) return;
  samp[k] = make_double4(uvw[3 * k], uvw[3 * k + 1], uvw[3 * k + 2], off ? off[k] : 0.0);
  if (ref4) {
    if (refs)
      ref4[k] = make_int4(checked_ref(refs[3 * k], G, badref), checked_ref(refs[3 * k + 1], G, badref),
                          checked_ref(refs[3 * k + 2], G, badref), -1);
    else
      ref4[k] = make_int4(-1, -1, -1, -1);
  }
}

// |u.s + off| bound check for the split path: max over samples of
// |u|+|v|+|w|+|off| (>= |u.s + off| for unit s).  Non-finite -> +inf.
__global__ void k_sample_bound(long long K, const double4 *samp, unsigned long long *out) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double b = 0;
  if (k < K) {
    const double4 s = samp[k];
    b = fabs(s.x) + fabs(s.y) + fabs(s.z) + fabs(s.w);
    if (!(b <= 1e300)) b = __longlong_as_double(0x7ff0000000000000ll);
  }
  for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(b)));
}

}  // namespace viss

namespace viss {

static inline unsigned nblk(long long n, int bs) { return static_cast<unsigned>((n + bs - 1) / bs); }

cudaError_t launch_occulters(long long n, const double *P, double R, int mode, double thr,
                             double4 *occ, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_occulters<<<nblk(n, 256), 256, 0, st>>>(n, P, R, mode, thr, occ);
  return cudaGetLastError();
}

cudaError_t launch_mask_bits(long long K, long long J, const double *lmn, const int32_t *refs,
                             const double4 *occ, uint32_t *bits, cudaStream_t st) {
  const long long words = K * ((J + 31) / 32);
  if (words <= 0) return cudaSuccess;
  k_mask_bits<<<nblk(words, 8), 256, 0, st>>>(K, J, lmn, refs, occ, bits);
  return cudaGetLastError();
}

cudaError_t launch_pix_keys(long long J, const double *lmn, unsigned long long *keys, int *idx,
                            cudaStream_t st) {
  if (J <= 0) return cudaSuccess;
  k_pix_keys<<<nblk(J, 256), 256, 0, st>>>(J, lmn, keys, idx);
  return cudaGetLastError();
}

cudaError_t launch_stage_pixels(long long J, long long Jpad, const double *lmn, const int *perm,
                                double4 *pix, float4 *cones, cudaStream_t st) {
  k_stage_pixels<<<nblk(Jpad, 256), 256, 0, st>>>(J, Jpad, lmn, perm, pix);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const long long nt = Jpad / kTilePix;
  k_tile_cones<<<nblk(nt, 8), 256, 0, st>>>(nt, pix, cones);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  k_super_cones<<<nblk((nt + kSuperTiles - 1) / kSuperTiles, 256), 256, 0, st>>>(nt, cones);
  return cudaGetLastError();
}

cudaError_t launch_occ32(long long G, const double4 *occ, float4 *out, cudaStream_t st) {
  if (G <= 0) return cudaSuccess;
  k_occ32<<<nblk(G, 256), 256, 0, st>>>(G, occ, out);
  return cudaGetLastError();
}

cudaError_t launch_stage_sky(long long J, long long Jpad, const double4 *pix, const int *perm,
                             const float *sky, float scale, double4 *out, int channels,
                             cudaStream_t st) {
  dim3 grid(nblk(Jpad, 256), static_cast<unsigned>(channels));
  k_stage_sky<<<grid, 256, 0, st>>>(J, Jpad, pix, perm, sky, scale, out);
  return cudaGetLastError();
}

// Coefficient staging for the adjoint: a 16-byte aligned copy padded to an
// even count (bulk copies move whole 16-byte units).
__global__ void k_stage_coef(long long K, long long Kpad, const float2 *coef, float2 *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= Kpad) return;
  out[i] = i < K ? coef[i] : make_float2(0.f, 0.f);
}

cudaError_t launch_stage_coef(long long K, long long Kpad, const float2 *coef, float2 *out,
                              cudaStream_t st) {
  if (Kpad <= 0) return cudaSuccess;
  k_stage_coef<<<nblk(Kpad, 256), 256, 0, st>>>(K, Kpad, coef, out);
  return cudaGetLastError();
}

cudaError_t launch_stage_samples(long long K, const double *uvw, const double *off,
                                 const int32_t *refs, long long G, double4 *samp, int4 *ref4,
                                 unsigned long long *bound, int *badref, cudaStream_t st) {
  if (K <= 0) return cudaSuccess;
  k_stage_samples<<<nblk(K, 256), 256, 0, st>>>(K, uvw, off, refs, G, samp, ref4, badref);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !bound) return e;
  k_sample_bound<<<nblk(K, 256), 256, 0, st>>>(K, samp, bound);
  return cudaGetLastError();
}

// Sort (key, index) pairs by key: the plan's pixel order.  Plan set-up only.
cudaError_t sort_pixel_keys(long long J, unsigned long long *keys_in, unsigned long long *keys_out,
                            int *idx_in, int *idx_out, cudaStream_t st) {
  size_t temp = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp, keys_in, keys_out, idx_in, idx_out,
                                                  static_cast<int>(J), 0, 50, st);
  if (e != cudaSuccess) return e;
  void *tmp = nullptr;
  e = cudaMallocAsync(&tmp, temp, st);
  if (e != cudaSuccess) return e;
  e = cub::DeviceRadixSort::SortPairs(tmp, temp, keys_in, keys_out, idx_in, idx_out,
                                      static_cast<int>(J), 0, 50, st);
  cudaError_t e2 = cudaFreeAsync(tmp, st);
  return e != cudaSuccess ? e : e2;
}

// Tile cones of already-staged pixel records (used by the allocation-free
// forward entry point, which stages pixels in the caller's order).
cudaError_t launch_tile_cones(long long ntiles, const double4 *pix, float4 *cones, cudaStream_t st) {
  if (ntiles <= 0) return cudaSuccess;
  k_tile_cones<<<nblk(ntiles, 8), 256, 0, st>>>(ntiles, pix, cones);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_super_cones<<<nblk((ntiles + kSuperTiles - 1) / kSuperTiles, 256), 256, 0, st>>>(ntiles, cones);
  return cudaGetLastError();
}

}  // namespace viss
