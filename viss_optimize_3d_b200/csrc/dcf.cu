// dcf.cu -- density compensation and per-row weights.
//
// Replaces the reference's shell pipeline
//   ceilAndScale     vissgen3d_blockage.cu:105-111  shell index per row
//   thrust::sort     vissgen3d_blockage.cu:456       (not needed for counting)
//   countOccurrences vissgen3d_blockage.cu:114-123  O(N*nr) loop, float atomics
//   calculateR       vissgen3d_blockage.cu:125-130
//   calculateDcf     vissgen3d_noblockage.cu:132-141 (the un-shifted formula;
//                    vissgen3d_blockage.cu:138 reads R[idx], mb[idx] one shell
//                    late and past the end at idx == nr)
// and the weight half of viss_gamma_trans (vissgen3d_blockage.cu:144-164)
// with the clamp of computeC (:178, :187).
//
// Counts are uint32 shared-memory histograms merged with integer atomics, so
// they are exact and order independent (the reference's float atomics stop
// counting exactly at 2^24 per shell).  Every floating-point step uses the
// _rn intrinsics so no FMA contraction changes a bit against the CPU oracle.
#include "viss_common.cuh"

namespace viss {

// Shell index, vissgen3d_blockage.cu:108: ceil((bll - 1/4) / 0.5) in FP32.
// NaN maps to -1 (no shell); magnitudes past 2^30 saturate.
__device__ __forceinline__ int shell_of(float bll) {
  const float c = ceilf(__fmul_rn(__fsub_rn(bll, 0.25f), 2.0f));
  if (!(c == c)) return -1;
  if (c > 1073741824.0f) return 1073741824;
  if (c < -1073741824.0f) return -1073741824;
  return static_cast<int>(c);
}

constexpr int kHistSmemBins = 12288;  // 48 KB of uint32 bins per CTA

__global__ void k_shell_hist(long long n, const float *bll, int nr, int32_t *gs,
                             unsigned int *counts) {
  extern __shared__ unsigned int s_hist[];
  const bool use_smem = nr <= kHistSmemBins;
  if (use_smem)
    for (int b = threadIdx.x; b < nr; b += blockDim.x) s_hist[b] = 0;
  __syncthreads();
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += stride) {
    const int g = shell_of(bll[i]);
    if (gs) gs[i] = g;
    if (g >= 1 && g <= nr) {
      if (use_smem) atomicAdd(&s_hist[g - 1], 1u);
      else atomicAdd(&counts[g - 1], 1u);
    }
  }
  __syncthreads();
  if (use_smem)
    for (int b = threadIdx.x; b < nr; b += blockDim.x)
      if (s_hist[b]) atomicAdd(&counts[b], s_hist[b]);
}

// dcf[0] = 1/(4 pi); dcf[k] = (2 pi/3)(R^3 - (R-1/2)^3) / (mult*counts[k-1]),
// R = k/2 + 1/4.  R^3 and (R-1/2)^3 are exact in FP64 for nr < 2^17.
__global__ void k_dcf_table(int nr, int mult, unsigned int *counts, float *dcf) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > nr) return;
  if (k == 0) {
    dcf[0] = static_cast<float>(1.0 / (4.0 * 3.141592653589793116));
    return;
  }
  if (mult != 1) counts[k - 1] *= static_cast<unsigned int>(mult);
  const double c = 2.0 * 3.141592653589793116 / 3.0;
  const double R = __dadd_rn(__dmul_rn(static_cast<double>(k), 0.5), 0.25);
  const double Rm = __dadd_rn(R, -0.5);
  const double vol = __dadd_rn(__dmul_rn(__dmul_rn(R, R), R), -__dmul_rn(__dmul_rn(Rm, Rm), Rm));
  dcf[k] = static_cast<float>(__ddiv_rn(__dmul_rn(c, vol), static_cast<double>(counts[k - 1])));
}

// dg and the clamped weight of each row.
__global__ void k_weights(long long n, const float *w, const float *bll, const int32_t *gs,
                          const float *dcf, int nr, float *dg_out, float *wt) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = __ddiv_rn(static_cast<double>(w[i]), static_cast<double>(bll[i]));
  float dg;
  if (!(fabs(x) < 1.0)) {
    dg = __int_as_float(0x7f800000);
  } else {
    const double x2 = __dmul_rn(x, x);
    const double num = __dmul_rn(1.5, __dsqrt_rn(fabs(__dadd_rn(1.0, -__dmul_rn(4.0, x2)))));
    dg = static_cast<float>(__ddiv_rn(num, __dsqrt_rn(__dadd_rn(1.0, -x2))));
  }
  if (dg_out) dg_out[i] = dg;
  if (wt) {
    int g = gs[i];
    g = g < 0 ? 0 : (g > nr ? nr : g);
    wt[i] = fminf(__fmul_rn(dcf[g], dg), 0.125f);
  }
}

// V <- V exp(-2 pi i w), phase in FP64 (vissgen3d_blockage.cu:150-151).
__global__ void k_wrot(long long n, const float *w, float2 *V) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double wd = static_cast<double>(w[i]);
  const double f = wd - rint(wd);
  double sn, cs;
  sincospi(2.0 * f, &sn, &cs);
  const float2 v = V[i];
  const double re = static_cast<double>(v.x), im = static_cast<double>(v.y);
  V[i] = make_float2(static_cast<float>(re * cs + im * sn), static_cast<float>(im * cs - re * sn));
}

// V[i + m] = conj(V[i]) for i < m (vissgen3d_blockage.cu:100).
__global__ void k_conj_mirror(long long m, float2 *V) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const float2 v = V[i];
  V[i + m] = make_float2(v.x, -v.y);
}

__global__ void k_scale_coef(long long n, const float *wt, const float2 *V, float2 *coef) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2 v = V[i];
  const float a = wt[i];
  coef[i] = make_float2(__fmul_rn(a, v.x), __fmul_rn(a, v.y));
}

}  // namespace viss

namespace viss {

static inline unsigned nblk2(long long n, int bs) { return static_cast<unsigned>((n + bs - 1) / bs); }

cudaError_t launch_dcf(long long n, const float *bll, int nr, int mult, int32_t *gs,
                       unsigned int *counts, float *dcf, int num_sms, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned int) * static_cast<size_t>(nr), st);
  if (e != cudaSuccess) return e;
  if (n > 0) {
    const size_t smem = nr <= kHistSmemBins ? sizeof(unsigned int) * static_cast<size_t>(nr) : 0;
    long long blocks = (n + 255) / 256;
    const long long cap = static_cast<long long>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    k_shell_hist<<<static_cast<unsigned>(blocks), 256, smem, st>>>(n, bll, nr, gs, counts);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  k_dcf_table<<<nblk2(nr + 1, 256), 256, 0, st>>>(nr, mult, counts, dcf);
  return cudaGetLastError();
}

cudaError_t launch_weights(long long n, const float *w, const float *bll, const int32_t *gs,
                           const float *dcf, int nr, float *dg, float *wt, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_weights<<<nblk2(n, 256), 256, 0, st>>>(n, w, bll, gs, dcf, nr, dg, wt);
  return cudaGetLastError();
}

cudaError_t launch_wrot(long long n, const float *w, float2 *V, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_wrot<<<nblk2(n, 256), 256, 0, st>>>(n, w, V);
  return cudaGetLastError();
}

cudaError_t launch_conj_mirror(long long m, float2 *V, cudaStream_t st) {
  if (m <= 0) return cudaSuccess;
  k_conj_mirror<<<nblk2(m, 256), 256, 0, st>>>(m, V);
  return cudaGetLastError();
}

cudaError_t launch_scale_coef(long long n, const float *wt, const float2 *V, float2 *coef,
                              cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  k_scale_coef<<<nblk2(n, 256), 256, 0, st>>>(n, wt, V, coef);
  return cudaGetLastError();
}

}  // namespace viss
