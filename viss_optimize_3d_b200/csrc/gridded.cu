// gridded.cu -- the unmasked imaging adjoint through per-facet type-3 NUFFTs.
//
//   image_j = scale * sum_k Re(coef_k exp(+2 pi i (u_k.s_j + off_k)))
//
// is the adjoint of the reference's noblockage programs, whose computeC has
// no occultation mask (vissgen3d_noblockage.cu:167-182).  Evaluated directly
// (k_adjoint) it costs K x J exponentials.  Here the sky is cut into facets:
// runs of the plan's pixel records, which are sorted by a hierarchical
// (NESTED) key, so a facet of 4^n records is a compact sky patch.  In the
// local frame of facet f (e3 = its centre direction c, e1 and e2 across it)
// a pixel is s = x e1 + y e2 + (1 + zc + z) e3 with |x|, |y| small and z
// tiny, so
//
//   u.s = nu1 x + nu2 y + nu3 z + nu3 (1 + zc),   nu = (u.e1, u.e2, u.e3),
//
// and the facet's image is a 3-D type-3 sum over the nonuniform frequencies
// nu_k and targets (x, y, z).  It is evaluated in three steps per facet:
//   1. spread c'_k = coef_k e^{2 pi i (nu3 (1 + zc) + off_k)} onto a uniform
//      nu-grid with the "exponential of semicircle" kernel
//      phi(t) = exp(beta (sqrt(1 - t^2) - 1)) (W points per dimension), each
//      contribution already multiplied by the grid point's (-1)^m / psi-hat;
//   2. transform the grid (cuFFT, C2C inverse);
//   3. interpolate the transform at each pixel's (x, y, z) with psi (W2
//      points per dimension) and divide by phi-hat there.
// Grid spacing h = 1 / (2 sigma X) per dimension for targets within |x| <= X,
// and M h >= 2 sigma2 (|u|max + W h / 2) points: the quadrature of step 2 is
// oversampled sigma = 2 times (W = 7), the interpolation of step 3 sigma2 =
// 1.5 times (W2 = 9, which keeps it as accurate as W2 = 7 at sigma2 = 2 with
// 2.4 times fewer grid points); ~1e-6 relative error per facet in FP64, FP32
// grids and transforms add a few 1e-7.  The grid is FP32 complex; positions on it are
// formed in FP64 and the phase offset nu3 (1 + zc) + off is reduced to a
// fraction of a turn in FP64 before its FP32 sincos.
//
// Spreading is the costly step (K W^3 grid updates per facet).  The samples
// are sorted once per call by a 3-D Morton key of u, so a block's 256
// consecutive samples lie close together in every facet's frame; the block
// accumulates them into a box of the grid in shared memory (fixed point, one
// warp per sample, lanes over the W^2 rows of its footprint, so the lanes of
// one atomic hit distinct cells) and adds the box to the grid in HBM once.  A
// block whose box does not fit falls back to atomics in HBM.
#include <cuda_runtime.h>
#include <cufft.h>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "viss_common.cuh"

namespace viss {

// Kernel parameters: beta = 0.97 pi (1 - 1 / (2 sigma)) W, the choice of
// Barnett, Magland and af Klinteberg (SIAM J. Sci. Comput. 41, 2019) for the
// "exponential of semicircle" kernel at oversampling sigma.
constexpr int kGridW = 7;                 // spreading kernel width (grid points per dimension)
constexpr double kGridBeta = 2.30 * kGridW;
constexpr double kGridSigma = 2.0;        // oversampling of the targets' extent
constexpr double kGridSigma2 = 1.5;       // oversampling of the FFT for the interpolation
constexpr int kInterpW = 9;               // interpolation kernel width at sigma2 = 1.5
constexpr double kInterpBeta = 0.97 * 3.14159265358979323846 * (1.0 - 1.0 / (2.0 * kGridSigma2)) * kInterpW;
constexpr int kPhiTable = 8192;           // phi-hat table entries per dimension
constexpr int kSpreadWarps = 8;
constexpr int kSpreadP = 32 * kSpreadWarps;   // samples per spreading block
constexpr int kBoxCells = 6016;               // shared-memory box capacity (complex points): 3 CTAs per SM
constexpr int kW3 = 3 * kGridW;               // kernel weights per sample
constexpr int kHybridAlign = 256;             // occulted plans: facets are whole direct-adjoint warp tiles
constexpr double kMixBitsMax = 2147483648.0;  // bytes of the mixed-pair bitmask at most
constexpr size_t kSpreadSmem = 2 * sizeof(float) * kBoxCells + sizeof(float) * kSpreadP * kW3 +
                               sizeof(int) * kSpreadP * 4 + sizeof(float2) * kSpreadP;

// A facet's local frame and extents (FP64).
struct FacetFrame {
  double e1[3], e2[3], c[3];
  double zc;            // centre of the facet's z-range
  double X[3];          // max |x|, max |y|, max |z - zc| over its pixels
};

// Grid shape shared by every facet of one call (from the largest extents).
struct GridGeom {
  int M[3];          // points per dimension (multiples of 4: the phase factors are +-1)
  double h[3];       // nu-grid spacing (wavelengths); nu_m = (m - M/2) h
  double dx[3];      // target-grid spacing, 1 / (M h); x_l = (l - M/2) dx
  double X[3];       // extents the phi-hat tables cover
};

__host__ __device__ inline double es_kernel(double t, double beta) {
  return fabs(t) < 1.0 ? exp(beta * (sqrt(1.0 - t * t) - 1.0)) : 0.0;
}

__device__ __forceinline__ float es_kernel_f(float t, float beta) {
  return fabsf(t) < 1.0f ? __expf(beta * (sqrtf(1.0f - t * t) - 1.0f)) : 0.0f;
}

namespace {

__device__ double block_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

__device__ double block_max(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = -1e300;
  for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) t = fmax(t, red[i]);
  return t;
}

// One block per facet: records [f * fp, min(J, (f + 1) * fp)) of the sorted
// pixel records.  Centre = normalised mean direction; e1, e2 complete a
// right-handed frame; then the extents of the local coordinates, also folded
// into xmax[0..2] (the bits of non-negative doubles order like the values).
//
// It also writes the facet's FP32 bounding cone (centre rounded to FP32, and
// the largest chord from it to a pixel plus the classification margin,
// rounded up; 4 for a facet whose mean direction is ~0, NaN if a pixel is
// NaN): the cone the occulted (hybrid) path classifies samples against.
__global__ void k_facet_frames(long long J, long long fp, const double4 *pix, FacetFrame *out,
                               unsigned long long *xmax, float4 *fcones) {
  __shared__ double red[32];
  const long long f = blockIdx.x;
  const long long r0 = f * fp, r1 = min(J, r0 + fp);
  double sx = 0, sy = 0, sz = 0;
  for (long long i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double4 p = pix[i];
    sx += p.x;
    sy += p.y;
    sz += p.z;
  }
  sx = block_sum(sx, red);
  sy = block_sum(sy, red);
  sz = block_sum(sz, red);
  double nrm = sqrt(sx * sx + sy * sy + sz * sz);
  double c[3] = {0.0, 0.0, 1.0};
  if (nrm > 0) c[0] = sx / nrm, c[1] = sy / nrm, c[2] = sz / nrm;
  const bool degenerate = !(nrm > 1e-6);
  const float4 cf = degenerate ? make_float4(1.f, 0.f, 0.f, 0.f)
                               : make_float4(__double2float_rn(c[0]), __double2float_rn(c[1]),
                                             __double2float_rn(c[2]), 0.f);
  // e1 = normalise(c x a) with a the axis least aligned with c
  double a[3] = {1.0, 0.0, 0.0};
  if (fabs(c[0]) > 0.9) a[0] = 0.0, a[1] = 1.0;
  double e1[3] = {c[1] * a[2] - c[2] * a[1], c[2] * a[0] - c[0] * a[2], c[0] * a[1] - c[1] * a[0]};
  nrm = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int d = 0; d < 3; ++d) e1[d] /= nrm;
  const double e2[3] = {c[1] * e1[2] - c[2] * e1[1], c[2] * e1[0] - c[0] * e1[2], c[0] * e1[1] - c[1] * e1[0]};
  double mx = 0, my = 0, zlo = 1e300, zhi = -1e300, rho = 0, nan_px = 0;
  for (long long i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    const double4 p = pix[i];
    const double dx = p.x - cf.x, dy = p.y - cf.y, dz = p.z - cf.z;
    rho = fmax(rho, sqrt(dx * dx + dy * dy + dz * dz));
    if (isnan(p.x) || isnan(p.y) || isnan(p.z)) nan_px = 1;
    mx = fmax(mx, fabs(p.x * e1[0] + p.y * e1[1] + p.z * e1[2]));
    my = fmax(my, fabs(p.x * e2[0] + p.y * e2[1] + p.z * e2[2]));
    const double z = p.x * c[0] + p.y * c[1] + p.z * c[2] - 1.0;
    zlo = fmin(zlo, z);
    zhi = fmax(zhi, z);
  }
  mx = block_max(mx, red);
  my = block_max(my, red);
  zhi = block_max(zhi, red);
  zlo = -block_max(-zlo, red);
  rho = block_max(rho, red);
  nan_px = block_max(nan_px, red);
  if (threadIdx.x == 0) {
    float4 cone = cf;
    cone.w = nan_px > 0 ? __int_as_float(0x7fc00000) : (degenerate ? 4.f : __double2float_ru(rho + kConeMargin32));
    fcones[f] = cone;
    FacetFrame fr;
    for (int d = 0; d < 3; ++d) fr.e1[d] = e1[d], fr.e2[d] = e2[d], fr.c[d] = c[d];
    fr.zc = 0.5 * (zlo + zhi);
    fr.X[0] = mx;
    fr.X[1] = my;
    fr.X[2] = 0.5 * (zhi - zlo);
    out[f] = fr;
    for (int d = 0; d < 3; ++d)
      atomicMax(xmax + d, static_cast<unsigned long long>(__double_as_longlong(fmax(fr.X[d], 0.0))));
  }
}

// max |u_k| over the staged samples, as the bits of a non-negative double.
__global__ void k_max_unorm(long long K, const double4 *samp, unsigned long long *out) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (k < K) {
    const double4 s = samp[k];
    v = sqrt(s.x * s.x + s.y * s.y + s.z * s.z);
  }
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(v)));
}

// 21 bits of x moved to every third bit (3-D Morton interleave).
__device__ __forceinline__ unsigned long long morton_spread(unsigned int x) {
  unsigned long long v = x & 0x1fffffu;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}

// Morton key of each sample's u, quantised over [-umax, umax]^3.
__global__ void k_sample_keys(long long K, const double4 *samp, double umax, unsigned long long *keys, int *idx) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const double4 s = samp[k];
  const double q = 0.5 * 2097151.0 / fmax(umax, 1e-300);
  const double u[3] = {s.x, s.y, s.z};
  unsigned long long key = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double v = fmin(fmax((u[d] + umax) * q, 0.0), 2097151.0);
    key |= morton_spread(static_cast<unsigned int>(v)) << d;
  }
  keys[k] = key;
  idx[k] = static_cast<int>(k);
}

// Coefficients alone in key order (the samples' order kept from an earlier call).
__global__ void k_gather_coef(long long K, const int *idx, const float2 *coef, float2 *cs) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k < K) cs[k] = coef[idx[k]];
}

// Samples, coefficients and (when given) occulter refs in key order.
__global__ void k_gather_samples(long long K, const int *idx, const double4 *samp, const float2 *coef,
                                 const int4 *refs, double4 *ss, float2 *cs, int4 *rs) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const int i = idx[k];
  ss[k] = samp[i];
  cs[k] = coef[i];
  if (refs) rs[k] = refs[i];
}

// round(a b) for |a b| < 2^22: a b + 1.5 2^23 lies in [2^23, 2^24), where
// FP32 spacing is 1, so the FMA itself rounds to the nearest integer.
__device__ __forceinline__ int round_small(float a, float b) {
  return __float_as_int(fmaf(a, b, 12582912.0f)) - 0x4B400000;
}

// Step 1: samples [b P, b P + P) of the key-ordered samples into facet f's
// grid, W^3 points each, every contribution times the point's pre-correction
// pre0[m0] pre1[m1] pre2[m2] = (-1)^m / psi-hat(nu_m).  With occulter refs
// (rs non-null) only the samples that see the whole facet (facet_open against
// its cone) are spread; the direct adjoint takes the others.
//
// Shared memory: the box as separate real and imaginary planes of 32-bit
// fixed-point sums (kBoxCells each), each sample's 3 W kernel weights, its
// first grid point (3 ints + a spare), its phased coefficient, and each warp's
// list of the block's samples to spread: 74 KB, so 3 blocks fit an SM (the
// measured best against 2 with a larger box and 4 with a smaller one, which
// sends more blocks to HBM).  Fixed point because integer adds
// are native shared-memory atomics (FP32 adds there are compare-and-swap
// loops): with the scale 4e6 / max_q max(|Re c_q|, |Im c_q|) over the block's
// samples every contribution is below 2^22 in magnitude (weights <= 1), so it
// is rounded to an integer by one FMA with 1.5 2^23 (no conversion
// instruction), and a box point, at most 256 contributions, stays below
// 2^30.  The step, 2.5e-7 of the block's largest coefficient, is below FP32
// rounding of the same accumulation (a running sum of several such terms).
// Box layout: point (a, b, l) at a P + b n2 + l with n2 odd and P = 7 n2
// (mod 32), so lane p = 7 i + j of a warp, which updates row (i, j) of a
// sample's footprint, hits bank p n2 (mod 32): the 32 lanes of every shared
// atomic fall in distinct banks.
__global__ void __launch_bounds__(kSpreadP, 3) k_spread(long long K, const double4 *ss, const float2 *cs, int use_off,
                                                        const int4 *rs, const float4 *occ32, const float4 *fcones,
                                                        const FacetFrame *frames, long long f, GridGeom g,
                                                        const float *pre0, const float *pre1, const float *pre2,
                                                        float2 *grid, int *status) {
  constexpr int W = kGridW;
  extern __shared__ __align__(16) unsigned char smem[];
  int *box_re = reinterpret_cast<int *>(smem);
  int *box_im = box_re + kBoxCells;
  float *wts = reinterpret_cast<float *>(box_im + kBoxCells);        // [P][3 W]
  int *m0s = reinterpret_cast<int *>(wts + kSpreadP * kW3);          // [P][4]
  float2 *cv = reinterpret_cast<float2 *>(m0s + kSpreadP * 4);       // [P]
  __shared__ int s_lo[3], s_hi[3];
  __shared__ float s_cmag[kSpreadWarps];
  __shared__ int s_count[kSpreadWarps];
  __shared__ unsigned char s_list[kSpreadP];                         // per warp: its samples to spread
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if (t < 3) s_lo[t] = INT_MAX, s_hi[t] = INT_MIN;
  __syncthreads();
  const FacetFrame &fr = frames[f];
  const long long k = static_cast<long long>(blockIdx.x) * kSpreadP + t;
  bool ok = k < K && (rs == nullptr || facet_open(rs[k], fcones[f], occ32));
  float cmag = 0.f;
  if (ok) {
    const double4 s = ss[k];
    const float2 a = cs[k];
    const double nu[3] = {s.x * fr.e1[0] + s.y * fr.e1[1] + s.z * fr.e1[2],
                          s.x * fr.e2[0] + s.y * fr.e2[1] + s.z * fr.e2[2],
                          s.x * fr.c[0] + s.y * fr.c[1] + s.z * fr.c[2]};
    // c' = coef e^{2 pi i (nu3 (1 + zc) + off)}, the phase reduced in FP64
    double ph = fma(nu[2], 1.0 + fr.zc, use_off ? s.w : 0.0);
    ph -= rint(ph);
    float sn, cs_;
    sincospif(2.0f * static_cast<float>(ph), &sn, &cs_);
    float2 c = make_float2(a.x * cs_ - a.y * sn, a.x * sn + a.y * cs_);
    if (!isfinite(c.x) || !isfinite(c.y)) {
      atomicOr(status, 4);
      ok = false;
    }
    cv[t] = c;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double gp = nu[d] / g.h[d] + 0.5 * g.M[d];       // (nu - nu_0) / h
      const int m = static_cast<int>(ceil(gp - 0.5 * W));
      if (m < 0 || m + W > g.M[d]) {
        if (ok) atomicOr(status, 1);
        ok = false;
      }
      m0s[t * 4 + d] = m;
      const float f0 = static_cast<float>(static_cast<double>(m) - gp);
#pragma unroll
      for (int i = 0; i < W; ++i)
        wts[t * kW3 + d * W + i] =
            es_kernel_f((f0 + static_cast<float>(i)) * (2.0f / W), static_cast<float>(kGridBeta));
    }
    if (ok) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        atomicMin(&s_lo[d], m0s[t * 4 + d]);
        atomicMax(&s_hi[d], m0s[t * 4 + d]);
      }
      cmag = fmaxf(fabsf(c.x), fabsf(c.y));
    }
  }
  // this warp's samples to spread, compacted
  const unsigned vb = __ballot_sync(0xffffffffu, ok);
  if (ok) s_list[warp * 32 + __popc(vb & ((1u << lane) - 1u))] = static_cast<unsigned char>(t);
  if (lane == 0) s_count[warp] = __popc(vb);
  for (int o = 16; o > 0; o >>= 1) cmag = fmaxf(cmag, __shfl_xor_sync(0xffffffffu, cmag, o));
  if (lane == 0) s_cmag[warp] = cmag;
  __syncthreads();
  if (s_lo[0] == INT_MAX) return;                  // nothing to spread in this block (uniform)
  float cmax = 0.f;
#pragma unroll
  for (int w = 0; w < kSpreadWarps; ++w) cmax = fmaxf(cmax, s_cmag[w]);
  if (!(cmax > 0.f)) return;                       // only zero coefficients (uniform)
  const float fx = 4.0e6f / cmax;                  // fixed-point scale: contributions below 2^22
  const float inv_fx = cmax / 4.0e6f;
  const int lo0 = s_lo[0], lo1 = s_lo[1], lo2 = s_lo[2];
  const long long n0l = s_hi[0] - lo0 + W, n1l = s_hi[1] - lo1 + W;
  const int n2r = s_hi[2] - lo2 + W;
  const int n2 = n2r | 1;
  const long long Pl = n1l * n2 + (((W * n2 - n1l * n2) % 32) + 32) % 32;   // >= n1 n2, = W n2 (mod 32)
  const bool in_box = n0l * Pl <= kBoxCells;       // uniform
  const int n1 = static_cast<int>(n1l), P = static_cast<int>(Pl), cells = static_cast<int>(n0l * Pl);
  if (in_box) {
    for (int c = t; c < cells; c += kSpreadP) box_re[c] = 0, box_im[c] = 0;
  } else if (t == 0) {
    atomicAdd(status + 1, 1);                      // blocks that spread into HBM directly
  }
  __syncthreads();
  const int count = s_count[warp];
  const long long M23 = static_cast<long long>(g.M[1]) * g.M[2];
  if (in_box) {
    // this lane's rows of a footprint: p = lane and p = lane + 32 (< W^2)
    const int ia = lane / W, ja = lane - ia * W;
    const int pb = lane + 32, ib = pb / W, jb = pb - ib * W;
    const bool has_b = pb < W * W;
    const int oa = ia * P + ja * n2, ob = ib * P + jb * n2;
#pragma unroll 2
    for (int i = 0; i < count; ++i) {
      const int q = s_list[warp * 32 + i];
      const int base = (m0s[q * 4] - lo0) * P + (m0s[q * 4 + 1] - lo1) * n2 + (m0s[q * 4 + 2] - lo2);
      const float2 c = cv[q];
      const float *wq = wts + q * kW3;
      float w2[W];
#pragma unroll
      for (int l = 0; l < W; ++l) w2[l] = wq[2 * W + l];
      {
        const float wij = wq[ia] * wq[W + ja] * fx;
        const float vr = c.x * wij, vi = c.y * wij;
        int *rr = box_re + base + oa, *ri = box_im + base + oa;
#pragma unroll
        for (int l = 0; l < W; ++l) {
          atomicAdd(rr + l, round_small(vr, w2[l]));
          atomicAdd(ri + l, round_small(vi, w2[l]));
        }
      }
      if (has_b) {
        const float wij = wq[ib] * wq[W + jb] * fx;
        const float vr = c.x * wij, vi = c.y * wij;
        int *rr = box_re + base + ob, *ri = box_im + base + ob;
#pragma unroll
        for (int l = 0; l < W; ++l) {
          atomicAdd(rr + l, round_small(vr, w2[l]));
          atomicAdd(ri + l, round_small(vi, w2[l]));
        }
      }
    }
  } else {
    for (int i = 0; i < count; ++i) {
      const int q = s_list[warp * 32 + i];
      const int q0 = m0s[q * 4], q1 = m0s[q * 4 + 1], q2 = m0s[q * 4 + 2];
      const float2 c = cv[q];
      const float *wq = wts + q * kW3;
      for (int p = lane; p < W * W; p += 32) {
        const int ii = p / W, j = p - (p / W) * W;
        const float wij = wq[ii] * wq[W + j];
        const float vr = c.x * wij, vi = c.y * wij;
        const float pij = pre0[q0 + ii] * pre1[q1 + j];
        float2 *row = grid + static_cast<long long>(q0 + ii) * M23 + static_cast<long long>(q1 + j) * g.M[2] + q2;
#pragma unroll
        for (int l = 0; l < W; ++l) {
          const float wl = wq[2 * W + l] * pij * pre2[q2 + l];
          atomicAdd(row + l, make_float2(vr * wl, vi * wl));
        }
      }
    }
    return;
  }
  __syncthreads();
  for (int c = t; c < cells; c += kSpreadP) {
    const int ir = box_re[c], ii = box_im[c];
    if (ir == 0 && ii == 0) continue;
    const float vr = static_cast<float>(ir) * inv_fx, vi = static_cast<float>(ii) * inv_fx;
    const int a = c / P;
    const int rem = c - a * P;
    const int b = rem / n2;
    const int l = rem - b * n2;
    if (b >= n1 || l >= n2r) continue;             // padding
    const int m0 = lo0 + a, m1 = lo1 + b, m2 = lo2 + l;
    const float fac = pre0[m0] * pre1[m1] * pre2[m2];
    atomicAdd(grid + static_cast<long long>(m0) * M23 + static_cast<long long>(m1) * g.M[2] + m2,
              make_float2(vr * fac, vi * fac));
  }
}

// phi-hat at x from a table over [-X, X] (kPhiTable points, linear).
__device__ __forceinline__ double phi_hat(const double *tab, double X, double x) {
  double u = (x + X) / (2.0 * X) * (kPhiTable - 1);
  u = fmin(fmax(u, 0.0), kPhiTable - 1.000001);
  const int i = static_cast<int>(u);
  const double f = u - i;
  return tab[i] + f * (tab[i + 1] - tab[i]);
}

// Step 3: the transform interpolated at each pixel of facet f (records
// [r0, r1)), divided by phi-hat; scale * Re into the image at the caller's
// pixel index.  The (-1)^l post-phase folds into the weights.
__global__ void k_interp(long long r0, long long r1, const double4 *pix, const int *perm,
                         const FacetFrame *frames, long long f, GridGeom g, const float2 *grid,
                         const double *tab0, const double *tab1, const double *tab2, double norm, float scale,
                         float *img, int accumulate, int *status) {
  constexpr int W = kInterpW;
  const long long i = r0 + static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= r1) return;
  const FacetFrame &fr = frames[f];
  const double4 p = pix[i];
  const double x[3] = {p.x * fr.e1[0] + p.y * fr.e1[1] + p.z * fr.e1[2],
                       p.x * fr.e2[0] + p.y * fr.e2[1] + p.z * fr.e2[2],
                       p.x * fr.c[0] + p.y * fr.c[1] + p.z * fr.c[2] - 1.0 - fr.zc};
  int l0[3];
  float f0[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double gp = x[d] / g.dx[d] + 0.5 * g.M[d];
    const int l = static_cast<int>(ceil(gp - 0.5 * W));
    if (l < 0 || l + W > g.M[d]) {
      atomicOr(status, 2);
      return;
    }
    l0[d] = l;
    f0[d] = static_cast<float>(static_cast<double>(l) - gp);
  }
  float w1[W], w2[W];
#pragma unroll
  for (int j = 0; j < W; ++j) {
    w1[j] = (((l0[1] + j) & 1) ? -1.0f : 1.0f) *
            es_kernel_f((f0[1] + static_cast<float>(j)) * (2.0f / W), static_cast<float>(kInterpBeta));
    w2[j] = (((l0[2] + j) & 1) ? -1.0f : 1.0f) *
            es_kernel_f((f0[2] + static_cast<float>(j)) * (2.0f / W), static_cast<float>(kInterpBeta));
  }
  const long long M23 = static_cast<long long>(g.M[1]) * g.M[2];
  float sr = 0.f;
#pragma unroll 1
  for (int a = 0; a < W; ++a) {
    const float wa = (((l0[0] + a) & 1) ? -1.0f : 1.0f) *
                     es_kernel_f((f0[0] + static_cast<float>(a)) * (2.0f / W), static_cast<float>(kInterpBeta));
    const float2 *plane =
        grid + static_cast<long long>(l0[0] + a) * M23 + static_cast<long long>(l0[1]) * g.M[2] + l0[2];
    float pa = 0.f;
#pragma unroll
    for (int b = 0; b < W; ++b) {
      const float2 *row = plane + static_cast<long long>(b) * g.M[2];
      float rr = 0.f;
#pragma unroll
      for (int c = 0; c < W; ++c) rr = fmaf(row[c].x, w2[c], rr);
      pa = fmaf(rr, w1[b], pa);
    }
    sr = fmaf(pa, wa, sr);
  }
  const double den = phi_hat(tab0, g.X[0], x[0]) * phi_hat(tab1, g.X[1], x[1]) * phi_hat(tab2, g.X[2], x[2]);
  double v = static_cast<double>(sr) * norm / den * static_cast<double>(scale);
  const long long j = perm[i];
  if (accumulate) v += static_cast<double>(img[j]);
  img[j] = static_cast<float>(v);
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton on P_n, FP64).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

// Transform of the kernel of half-width a and parameter beta at frequency f:
// int_{-a}^{a} phi(t / a) cos(2 pi f t) dt.
double kernel_ft(double a, double beta, double f, const std::vector<double> &gx, const std::vector<double> &gw) {
  double s = 0.0;
  for (size_t i = 0; i < gx.size(); ++i)
    s += gw[i] * es_kernel(gx[i], beta) * std::cos(2.0 * M_PI * f * a * gx[i]);
  return s * a;
}

// Occulted plans: of nsub samples (every stride-th) x nF facets, the pairs
// whose facet is wholly visible (counts[0]) and those neither wholly visible
// nor wholly hidden (counts[1], the direct kernel's share).
__global__ void k_count_states(long long nsub, long long stride, const int4 *refs, const float4 *occ32,
                               const float4 *fcones, long long nF, unsigned long long *counts) {
  unsigned long long open = 0, mixed = 0;
  const long long n = nsub * nF;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long k = (i / nF) * stride, f = i - (i / nF) * nF;
    const int4 rf = refs[k];
    const float4 cone = fcones[f];
    if (facet_open(rf, cone, occ32)) {
      ++open;
      continue;
    }
    bool hidden = false;
    const int r3[3] = {rf.x, rf.y, rf.z};
    for (int c = 0; c < 3; ++c) hidden = hidden || (r3[c] >= 0 && cone_state32(cone, occ32[r3[c]]) == 0);
    if (!hidden) ++mixed;
  }
  for (int o = 16; o > 0; o >>= 1) {
    open += __shfl_xor_sync(0xffffffffu, open, o);
    mixed += __shfl_xor_sync(0xffffffffu, mixed, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counts, open);
    atomicAdd(counts + 1, mixed);
  }
}

// Occulted plans: bit (k mod 32) of mixbits[f * words + k / 32] is set iff
// sample k (original order) neither sees facet f wholly (facet_open) nor is
// hidden on all of it (a row classifies the cone as hidden): the pairs the
// direct kernel must evaluate.  One warp per 32 samples, its rows loaded
// once and tested against every facet's cone.
__global__ void k_mixed_bits(long long K, long long nF, long long words, const int4 *refs, const float4 *occ32,
                             const float4 *fcones, unsigned *mixbits) {
  const long long w = static_cast<long long>(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
  if (w >= words) return;                                            // uniform over the warp
  const int lane = threadIdx.x & 31;
  const long long k = w * 32 + lane;
  const float4 pass32 = make_float4(0.f, 0.f, 0.f, -4.f);
  int4 rf = make_int4(-1, -1, -1, -1);
  if (k < K) rf = refs[k];
  const float4 r0 = rf.x >= 0 ? occ32[rf.x] : pass32, r1 = rf.y >= 0 ? occ32[rf.y] : pass32,
               r2 = rf.z >= 0 ? occ32[rf.z] : pass32;
  for (long long f = 0; f < nF; ++f) {
    const float4 cone = fcones[f];
    const int s0 = cone_state32(cone, r0), s1 = cone_state32(cone, r1), s2 = cone_state32(cone, r2);
    const bool open = (rf.x < 0 || s0 == 2) && (rf.y < 0 || s1 == 2) && (rf.z < 0 || s2 == 2);
    const bool hidden = (rf.x >= 0 && s0 == 0) || (rf.y >= 0 && s1 == 0) || (rf.z >= 0 && s2 == 0);
    const unsigned b = __ballot_sync(0xffffffffu, k < K && !open && !hidden);
    if (lane == 0) mixbits[f * words + w] = b;
  }
}

// The smallest n >= m with n % 4 == 0 and no prime factor above 7 (FFT-friendly).
int fft_size(long long m) {
  for (long long n = std::max<long long>(4, (m + 3) / 4 * 4);; n += 4) {
    long long r = n;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return static_cast<int>(n);
  }
}

}  // namespace

// Device buffers and the FFT plan, kept between calls on one viss_plan.
struct GriddedState {
  float2 *grid = nullptr;
  size_t grid_cap = 0;
  cufftHandle fft = 0;
  int fft_dims[3] = {0, 0, 0};
  bool fft_ok = false;
  FacetFrame *frames = nullptr;
  size_t frames_cap = 0;
  float4 *fcones = nullptr;        // facet bounding cones (FP32, as the tile cones)
  size_t fcones_cap = 0;
  int4 *rs = nullptr;              // occulter refs in key order (occulted plans)
  size_t rs_cap = 0;
  unsigned *mixbits = nullptr;     // occulted plans: the (sample, facet) pairs left to the direct kernel
  size_t mixbits_cap = 0;
  float *pre = nullptr;            // pre0 | pre1 | pre2
  size_t pre_cap = 0;
  double *tabs = nullptr;          // 3 x kPhiTable
  GridGeom tab_geom{};             // the grid the tables in pre / tabs were made for
  bool tabs_valid = false;
  int *status = nullptr;           // [0] flags (1, 2: footprint left the grid, 4: non-finite coefficient),
                                   // [1] blocks spread into HBM directly
  unsigned long long *red = nullptr;   // max extents (3) and max |u| (1), as double bits
  unsigned char *sort = nullptr;   // keys (2 K), indices (2 K), radix-sort temporaries
  size_t sort_cap = 0;
  double4 *ss = nullptr;           // samples in key order
  size_t ss_cap = 0;
  float2 *cs = nullptr;            // coefficients in key order
  size_t cs_cap = 0;
  // what the last successful call derived from the plan's geometry alone (the
  // |u| bound, the facet size and extents, the sample order, the mixed-pair
  // bits), reused while the plan's geometry version and the request match
  long long cache_version = -1, cache_request = -1, cache_fp = 0, cache_words = 0;
  bool cache_masked = false, cache_mix = false;
  double cache_umax = 0, cache_X[3] = {0, 0, 0};
  ~GriddedState() {
    if (fft_ok) cufftDestroy(fft);
    void *bufs[] = {grid, frames, fcones, rs, mixbits, pre, tabs, status, red, sort, ss, cs};
    for (void *b : bufs)
      if (b) cudaFree(b);
  }
};

void gridded_free(void *state) { delete static_cast<GriddedState *>(state); }

int record_error(int status, const std::string &msg);

namespace {
template <class T>
bool grow(T *&p, size_t &cap, size_t bytes) {
  if (p && bytes <= cap) return true;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  if (cudaMalloc(reinterpret_cast<void **>(&p), bytes) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cap = bytes;
  return true;
}
int cuda_err(cudaError_t e, const char *where) {
  return record_error(-2, std::string("viss_adjoint_gridded: ") + where + ": " + cudaGetErrorString(e));
}

// Modelled seconds per grid update of the spreading step and per grid point
// of a facet's memset + FFT (B200, FP32 complex grid); they only rank the
// candidate facet sizes.
constexpr double kSecPerUpdate = 6.5e-13;
constexpr double kSecPerCell = 1.6e-11;
// and per (sample, pixel) pair of a mixed facet left to the direct kernel
// (tile culling inside the facet included)
constexpr double kSecPerMixedPair = 3.0e-13;

// Grid shape for targets within |x_d| <= X[d] and |u| <= umax.
GridGeom grid_geom(const double X_in[3], double umax) {
  GridGeom g;
  for (int d = 0; d < 3; ++d) {
    const double X = std::max(X_in[d] * (1.0 + 1e-9), 1e-9);
    g.X[d] = X;
    g.h[d] = 1.0 / (2.0 * kGridSigma * X);
    const double up = umax * (1.0 + 1e-12) + 0.5 * kGridW * g.h[d];
    const long long need = static_cast<long long>(std::ceil(2.0 * kGridSigma2 * up / g.h[d])) + 2;
    // the targets fill the central half: an interpolation footprint needs M / 4 >= W2 / 2 + 1
    g.M[d] = fft_size(std::max<long long>(need, 2 * kInterpW + 6));
    g.dx[d] = 1.0 / (g.M[d] * g.h[d]);
  }
  return g;
}

bool same_grid(const GridGeom &a, const GridGeom &b) {
  for (int d = 0; d < 3; ++d)
    if (a.M[d] != b.M[d] || a.h[d] != b.h[d] || a.dx[d] != b.dx[d] || a.X[d] != b.X[d]) return false;
  return true;
}

double grid_cells(const GridGeom &g) { return static_cast<double>(g.M[0]) * g.M[1] * g.M[2]; }

// Frames of the facets of fp records into S.frames; their largest extents
// into X (one device round trip).
int facet_frames(GriddedState &S, long long J, long long fp, const double4 *pix, cudaStream_t st, double X[3]) {
  const long long nF = (J + fp - 1) / fp;
  if (!grow(S.frames, S.frames_cap, sizeof(FacetFrame) * nF) || !grow(S.fcones, S.fcones_cap, sizeof(float4) * nF))
    return record_error(-3, "viss_adjoint_gridded: device allocation failed (facet frames)");
  cudaError_t e;
  if ((e = cudaMemsetAsync(S.red, 0, 3 * sizeof(unsigned long long), st)) != cudaSuccess) return cuda_err(e, "memset");
  k_facet_frames<<<static_cast<unsigned>(nF), 256, 0, st>>>(J, fp, pix, S.frames, S.red, S.fcones);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "frames");
  unsigned long long b[3];
  if ((e = cudaMemcpyAsync(b, S.red, sizeof(b), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_err(e, "read back");
  for (int d = 0; d < 3; ++d) std::memcpy(&X[d], &b[d], sizeof(double));
  return 0;
}

// Shares of wholly visible and of mixed (sample, facet) pairs over the nF
// facets whose cones are in S.fcones, from up to 2,048 evenly spaced samples.
int pair_shares(GriddedState &S, long long K, const int4 *refs, const float4 *occ32, long long nF, cudaStream_t st,
                double &open, double &mixed) {
  const long long nsub = std::min<long long>(K, 2048), stride = K / nsub;
  cudaError_t e;
  if ((e = cudaMemsetAsync(S.red + 4, 0, 2 * sizeof(unsigned long long), st)) != cudaSuccess) return cuda_err(e, "memset");
  k_count_states<<<592, 256, 0, st>>>(nsub, stride, refs, occ32, S.fcones, nF, S.red + 4);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "pair shares");
  unsigned long long c[2];
  if ((e = cudaMemcpyAsync(c, S.red + 4, sizeof(c), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_err(e, "read back");
  const double n = static_cast<double>(nsub) * nF;
  open = c[0] / n;
  mixed = c[1] / n;
  return 0;
}

// The samples and coefficients in the Morton order of u, into S.ss / S.cs.
int sort_samples(GriddedState &S, long long K, const double4 *samp, const float2 *coef, const int4 *refs,
                 double umax, cudaStream_t st) {
  size_t temp = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp, static_cast<unsigned long long *>(nullptr),
                                                  static_cast<unsigned long long *>(nullptr),
                                                  static_cast<int *>(nullptr), static_cast<int *>(nullptr),
                                                  static_cast<int>(K), 0, 63, st);
  if (e != cudaSuccess) return cuda_err(e, "sort size");
  const size_t keys_b = sizeof(unsigned long long) * K, idx_b = sizeof(int) * K;
  const size_t off_idx = 2 * keys_b, off_tmp = (off_idx + 2 * idx_b + 255) / 256 * 256;
  if (!grow(S.sort, S.sort_cap, off_tmp + temp) || !grow(S.ss, S.ss_cap, sizeof(double4) * K) ||
      !grow(S.cs, S.cs_cap, sizeof(float2) * K) || (refs && !grow(S.rs, S.rs_cap, sizeof(int4) * K)))
    return record_error(-3, "viss_adjoint_gridded: device allocation failed (sample order)");
  auto *keys = reinterpret_cast<unsigned long long *>(S.sort);
  auto *idx = reinterpret_cast<int *>(S.sort + off_idx);
  const unsigned nb = static_cast<unsigned>((K + 255) / 256);
  k_sample_keys<<<nb, 256, 0, st>>>(K, samp, umax, keys, idx);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "sample keys");
  if ((e = cub::DeviceRadixSort::SortPairs(S.sort + off_tmp, temp, keys, keys + K, idx, idx + K, static_cast<int>(K),
                                           0, 63, st)) != cudaSuccess)
    return cuda_err(e, "sort");
  k_gather_samples<<<nb, 256, 0, st>>>(K, idx + K, samp, coef, refs, S.ss, S.cs, S.rs);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "gather samples");
  return 0;
}
}  // namespace

// image (J, caller's order) = scale * Re(unmasked adjoint) through facets of
// `facet_pix` sorted records (0: the candidate 4^n, n >= 3, with the least
// modelled time whose grid holds at most max_cells points; the choice is
// returned in *facet_used).  samp / coef are the plan's staged samples and
// coefficients.  info[0] = blocks that spread into HBM directly, summed over
// the facets.  Returns a viss status (0 = ok).
int gridded_adjoint(void **statep, long long J, const double4 *pix, const int *perm, long long K,
                    const double4 *samp, const float2 *coef, int use_off, long long facet_pix,
                    float scale, float *img, int accumulate, long long max_cells, cudaStream_t st,
                    int *grid_dims, long long *facet_used, long long *info, const int4 *refs,
                    const float4 *occ32, const float4 **fcones_out, const unsigned **mixbits_out,
                    long long *mix_words_out, long long geom_version) {
  if (K > INT_MAX) return record_error(-1, "viss_adjoint_gridded: more than 2^31 - 1 samples");
  const bool masked = refs != nullptr;
  if (masked && facet_pix % kHybridAlign != 0)
    return record_error(-1, "viss_adjoint_gridded: with occultation, facet_pixels must be a multiple of " +
                                std::to_string(kHybridAlign));
  if (!*statep) *statep = new GriddedState();
  GriddedState &S = *static_cast<GriddedState *>(*statep);
  if ((!S.tabs && cudaMalloc(&S.tabs, sizeof(double) * 3 * kPhiTable) != cudaSuccess) ||
      (!S.status && cudaMalloc(&S.status, 2 * sizeof(int)) != cudaSuccess) ||
      (!S.red && cudaMalloc(&S.red, 6 * sizeof(unsigned long long)) != cudaSuccess))
    return record_error(-3, "viss_adjoint_gridded: device allocation failed");
  cudaError_t e;
  if ((e = cudaMemsetAsync(S.red + 3, 0, sizeof(unsigned long long), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(S.status, 0, 2 * sizeof(int), st)) != cudaSuccess)
    return cuda_err(e, "memset");
  const bool cached = geom_version >= 0 && S.cache_version == geom_version && S.cache_request == facet_pix &&
                      S.cache_masked == masked;
  S.cache_version = -1;   // set again only when this call succeeds
  double umax = S.cache_umax;
  if (!cached) {
    k_max_unorm<<<static_cast<unsigned>((K + 255) / 256), 256, 0, st>>>(K, samp, S.red + 3);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "max |u|");
    unsigned long long ub = 0;
    if ((e = cudaMemcpyAsync(&ub, S.red + 3, sizeof(ub), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return cuda_err(e, "read back");
    std::memcpy(&umax, &ub, sizeof(umax));
    if (!std::isfinite(umax)) return record_error(-5, "viss_adjoint_gridded: non-finite uvw");
  }

  double X[3] = {S.cache_X[0], S.cache_X[1], S.cache_X[2]};
  long long fp = cached ? S.cache_fp : facet_pix;
  if (cached) {
    // frames, cones, sorted samples and mixed-pair bits are those of the last call
  } else if (fp == 0) {
    // every candidate's real extents (and, with occultation, its share of
    // wholly visible and of mixed sample-facet pairs), then the least
    // modelled time
    double best_t = 1e300;
    long long last = 0;
    for (long long c = masked ? kHybridAlign : 64;; c *= 4) {
      if (int s = facet_frames(S, J, c, pix, st, X)) return s;
      last = c;
      const double cells = grid_cells(grid_geom(X, umax));
      if (cells <= static_cast<double>(max_cells)) {
        const double nf = std::ceil(static_cast<double>(J) / c);
        double open = 1.0, mixed = 0.0;
        if (masked)
          if (int s = pair_shares(S, K, refs, occ32, static_cast<long long>(nf), st, open, mixed)) return s;
        const double t = nf * (static_cast<double>(K) * open * kGridW * kGridW * kGridW * kSecPerUpdate +
                               cells * kSecPerCell) +
                         static_cast<double>(K) * J * mixed * kSecPerMixedPair;
        if (t < best_t) best_t = t, fp = c;
      }
      if (c >= J) break;
    }
    if (fp == 0) return record_error(-1, "viss_adjoint_gridded: no facet size keeps the grid under its limit");
    if (fp != last)
      if (int s = facet_frames(S, J, fp, pix, st, X)) return s;
  } else if (int s = facet_frames(S, J, fp, pix, st, X)) {
    return s;
  }
  if (facet_used) *facet_used = fp;
  if (fcones_out) *fcones_out = S.fcones;
  if (mixbits_out) *mixbits_out = nullptr;
  bool mix_ok = false;
  const long long words = (K + 31) / 32;
  if (masked && cached) {
    mix_ok = S.cache_mix;
    if (mix_ok && mixbits_out) *mixbits_out = S.mixbits;
    if (mix_ok && mix_words_out) *mix_words_out = S.cache_words;
  } else if (masked) {
    // the pairs the direct kernel evaluates, once per geometry (up to 2 GiB
    // of bits; beyond that the direct kernel classifies each pair itself)
    const long long nF = (J + fp - 1) / fp;
    const double bytes = static_cast<double>(nF) * words * sizeof(unsigned);
    if (bytes <= kMixBitsMax && mixbits_out) {
      if (!grow(S.mixbits, S.mixbits_cap, static_cast<size_t>(bytes)))
        return record_error(-3, "viss_adjoint_gridded: device allocation failed (mixed-pair bits)");
      k_mixed_bits<<<static_cast<unsigned>((words + 7) / 8), 256, 0, st>>>(K, nF, words, refs, occ32, S.fcones,
                                                                           S.mixbits);
      if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "mixed-pair bits");
      *mixbits_out = S.mixbits;
      if (mix_words_out) *mix_words_out = words;
      mix_ok = true;
    }
  }
  const long long nF = (J + fp - 1) / fp;
  // one grid shape for every facet, from the largest extents
  const GridGeom g = grid_geom(X, umax);
  const long long cells = static_cast<long long>(g.M[0]) * g.M[1] * g.M[2];
  if (grid_dims)
    for (int d = 0; d < 3; ++d) grid_dims[d] = g.M[d];
  if (cells > max_cells)
    return record_error(-1, "viss_adjoint_gridded: the facet grid would hold " + std::to_string(cells) +
                                " points (" + std::to_string(g.M[0]) + " x " + std::to_string(g.M[1]) + " x " +
                                std::to_string(g.M[2]) + "), above the limit; use smaller facets");
  // kernel transforms: pre[d][m] = (-1)^m / psi-hat(nu_m), phi-hat tables
  // (kept while the grid stays the same)
  if (!grow(S.grid, S.grid_cap, sizeof(float2) * cells))
    return record_error(-3, "viss_adjoint_gridded: device allocation failed (grid of " + std::to_string(cells) +
                                " points)");
  if (!S.tabs_valid || !same_grid(S.tab_geom, g)) {
    S.tabs_valid = false;
    std::vector<double> gx, gw;
    gauss_legendre(96, gx, gw);
    std::vector<float> pre(static_cast<size_t>(g.M[0]) + g.M[1] + g.M[2]);
    std::vector<double> tab(3 * static_cast<size_t>(kPhiTable));
    size_t o = 0;
    for (int d = 0; d < 3; ++d) {
      const double a_psi = 0.5 * kInterpW * g.dx[d], a_phi = 0.5 * kGridW * g.h[d];
      for (int m = 0; m < g.M[d]; ++m) {
        const double nu = (m - 0.5 * g.M[d]) * g.h[d];
        pre[o++] = static_cast<float>(((m & 1) ? -1.0 : 1.0) / kernel_ft(a_psi, kInterpBeta, nu, gx, gw));
      }
      for (int i = 0; i < kPhiTable; ++i) {
        const double x = -g.X[d] + 2.0 * g.X[d] * i / (kPhiTable - 1);
        tab[d * kPhiTable + i] = kernel_ft(a_phi, kGridBeta, x, gx, gw);
      }
    }
    if (!grow(S.pre, S.pre_cap, sizeof(float) * pre.size()))
      return record_error(-3, "viss_adjoint_gridded: device allocation failed (tables)");
    // synchronous copies: the host vectors go out of scope here
    if ((e = cudaMemcpyAsync(S.pre, pre.data(), sizeof(float) * pre.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(S.tabs, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
      return cuda_err(e, "tables");
    S.tab_geom = g;
    S.tabs_valid = true;
  }
  if (!S.fft_ok || S.fft_dims[0] != g.M[0] || S.fft_dims[1] != g.M[1] || S.fft_dims[2] != g.M[2]) {
    if (S.fft_ok) cufftDestroy(S.fft);
    S.fft_ok = false;
    if (cufftPlan3d(&S.fft, g.M[0], g.M[1], g.M[2], CUFFT_C2C) != CUFFT_SUCCESS)
      return record_error(-3, "viss_adjoint_gridded: cufftPlan3d failed");
    S.fft_ok = true;
    for (int d = 0; d < 3; ++d) S.fft_dims[d] = g.M[d];
  }
  if (cufftSetStream(S.fft, st) != CUFFT_SUCCESS) return record_error(-2, "viss_adjoint_gridded: cufftSetStream failed");
  if (cached) {
    const int *idx = reinterpret_cast<const int *>(S.sort + 2 * sizeof(unsigned long long) * K) + K;
    k_gather_coef<<<static_cast<unsigned>((K + 255) / 256), 256, 0, st>>>(K, idx, coef, S.cs);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "gather coefficients");
  } else if (int s = sort_samples(S, K, samp, coef, refs, umax, st)) {
    return s;
  }
  if ((e = cudaFuncSetAttribute(k_spread, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kSpreadSmem))) != cudaSuccess)
    return cuda_err(e, "spread attributes");
  const double norm = 1.0 / static_cast<double>(cells);
  const float *pre0 = S.pre, *pre1 = S.pre + g.M[0], *pre2 = S.pre + g.M[0] + g.M[1];
  const unsigned spread_blocks = static_cast<unsigned>((K + kSpreadP - 1) / kSpreadP);
  for (long long f = 0; f < nF; ++f) {
    const long long r0 = f * fp, r1 = std::min(J, r0 + fp);
    if ((e = cudaMemsetAsync(S.grid, 0, sizeof(float2) * cells, st)) != cudaSuccess) return cuda_err(e, "memset");
    k_spread<<<spread_blocks, kSpreadP, kSpreadSmem, st>>>(K, S.ss, S.cs, use_off, masked ? S.rs : nullptr, occ32,
                                                           S.fcones, S.frames, f, g, pre0, pre1, pre2, S.grid,
                                                           S.status);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "spread");
    if (cufftExecC2C(S.fft, reinterpret_cast<cufftComplex *>(S.grid), reinterpret_cast<cufftComplex *>(S.grid),
                     CUFFT_INVERSE) != CUFFT_SUCCESS)
      return record_error(-2, "viss_adjoint_gridded: cufftExecC2C failed");
    k_interp<<<static_cast<unsigned>((r1 - r0 + 127) / 128), 128, 0, st>>>(
        r0, r1, pix, perm, S.frames, f, g, S.grid, S.tabs, S.tabs + kPhiTable, S.tabs + 2 * kPhiTable, norm, scale,
        img, accumulate, S.status);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(e, "interpolate");
  }
  int status[2] = {0, 0};
  if ((e = cudaMemcpyAsync(status, S.status, sizeof(status), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
      (e = cudaStreamSynchronize(st)) != cudaSuccess)
    return cuda_err(e, "status");
  if (info) info[0] = status[1];
  if (status[0] & 4) return record_error(-5, "viss_adjoint_gridded: non-finite coefficients");
  if (status[0]) return record_error(-2, "viss_adjoint_gridded: a kernel footprint left the grid (internal error)");
  S.cache_version = geom_version;
  S.cache_request = facet_pix;
  S.cache_masked = masked;
  S.cache_fp = fp;
  S.cache_umax = umax;
  for (int d = 0; d < 3; ++d) S.cache_X[d] = X[d];
  S.cache_mix = mix_ok;
  S.cache_words = words;
  return 0;
}

}  // namespace viss
