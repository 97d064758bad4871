// days.cu -- per-day staging and multi-day accumulation for the streaming day
// loop (host/vissgen_stream_main.cpp).
//
//   viss_stage_day_rows    one day's FP32 rows (the reference's uvw / xyza /
//                          xyzb / bll files, vissgen3d_blockage.cu:309-391)
//                          -> the FP64 geometry the plan takes, on the device
//                          instead of in host loops
//   viss_accumulate_image  sum[j] += img[j] in FP64, non-finite pixels as 0:
//                          the notebooks' day sum (healpix3d_blockage.ipynb:
//                          103-116), done on the device
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "viss.h"

namespace viss {
int record_error(int status, const std::string &msg);
}

namespace {

inline unsigned nblk(long long n, int bs) { return static_cast<unsigned>((n + bs - 1) / bs); }

// Row i of a day (n rows: the unique samples, then their mirrors):
//   uvw[i]  = (u, v, w)                          FP64 copy of the FP32 row
//   off[i]  = -w                                 the forward's w(n-1) term
//   P[i]    = satellite a, P[n + i] = satellite b (occulter rows i and n + i)
//   refs[i] = (i, n + i, -1)
//   w[i]    = w (FP32), bll kept as given
__global__ void k_stage_day_rows(long long n, const float *uvw3, const float *xa3,
                                 const float *xb3, double *uvw, double *off, double *P,
                                 int32_t *refs, float *w) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float u = uvw3[3 * i], v = uvw3[3 * i + 1], ww = uvw3[3 * i + 2];
  uvw[3 * i] = u;
  uvw[3 * i + 1] = v;
  uvw[3 * i + 2] = ww;
  off[i] = -static_cast<double>(ww);
  P[3 * i] = xa3[3 * i];
  P[3 * i + 1] = xa3[3 * i + 1];
  P[3 * i + 2] = xa3[3 * i + 2];
  P[3 * (n + i)] = xb3[3 * i];
  P[3 * (n + i) + 1] = xb3[3 * i + 1];
  P[3 * (n + i) + 2] = xb3[3 * i + 2];
  refs[3 * i] = static_cast<int32_t>(i);
  refs[3 * i + 1] = static_cast<int32_t>(n + i);
  refs[3 * i + 2] = -1;
  w[i] = ww;
}

__global__ void k_accumulate_image(long long n, const float *img, double *sum) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = img[i];
  sum[i] += isfinite(x) ? static_cast<double>(x) : 0.0;
}

int cuda_fail(cudaError_t e, const char *who) {
  return viss::record_error(VISS_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int viss_stage_day_rows(int64_t n, const float *uvw3, const float *xyza3, const float *xyzb3,
                        double *uvw, double *off, double *P, int32_t *refs, float *w,
                        void *stream) {
  if (n < 0 || (n > 0 && (!uvw3 || !xyza3 || !xyzb3 || !uvw || !off || !P || !refs || !w)))
    return viss::record_error(VISS_ERR_ARG, "viss_stage_day_rows: bad arguments");
  if (n >= (1LL << 30))
    return viss::record_error(VISS_ERR_ARG, "viss_stage_day_rows: too many rows for int32 refs");
  if (n == 0) return VISS_OK;
  k_stage_day_rows<<<nblk(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      n, uvw3, xyza3, xyzb3, uvw, off, P, refs, w);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VISS_OK : cuda_fail(e, "viss_stage_day_rows");
}

int viss_accumulate_image(int64_t n, const float *img, double *sum, void *stream) {
  if (n < 0 || (n > 0 && (!img || !sum)))
    return viss::record_error(VISS_ERR_ARG, "viss_accumulate_image: bad arguments");
  if (n == 0) return VISS_OK;
  k_accumulate_image<<<nblk(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(n, img, sum);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VISS_OK : cuda_fail(e, "viss_accumulate_image");
}

}  // extern "C"
