// vissgen_main.cpp -- drop-in replacement for the reference executables
// vissgen3d_blockage, vissgen3d_blockage_10m, vissgen3d_noblockage and
// vissgen3d_noblockage_10m (one source, four builds):
//
//   VISS_VARIANT_BLOCKAGE  1: occultation mask in imaging too
//                          (vissgen3d_blockage.cu:180-186); 0: forward only
//                          (vissgen3d_noblockage.cu:167-182)
//   VISS_VARIANT_10M       1: ./earth_10Mhz/*_10Mhz.txt inputs, 1 day, 10 MHz,
//                          one GPU (vissgen3d_blockage_10m.cu:50,199-219,568)
//
// Same command line (no arguments), same CWD-relative inputs and output
// directory, same stdout skeleton as the reference's vissGen
// (vissgen3d_blockage.cu:195-563).  The GPU work goes through libviss
// (include/viss.h).  Optional flags (not in the reference):
//   --days N       number of days (default 450, or 1 for the 10 MHz builds)
//   --first-day D  first day index, 1-based (default 1)
//   --data-dir P   input directory (default ./earth_1Mhz/ or ./earth_10Mhz/)
//   --out-dir P    output directory (default 3dblockage/ etc.)
//   --fp64         the plain FP64 path instead of split precision
//   --devices N    at most N GPUs (default: all)
// Days are spread round-robin over the GPUs, one host thread per GPU, like
// the reference's OpenMP loop (vissgen3d_blockage.cu:271-279); file reads and
// writes are serialised (its omp critical sections, :309, :535).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "textio.h"
#include "viss.h"

#ifndef VISS_VARIANT_BLOCKAGE
#define VISS_VARIANT_BLOCKAGE 1
#endif
#ifndef VISS_VARIANT_10M
#define VISS_VARIANT_10M 0
#endif

using viss_host::read_rows1;
using viss_host::read_rows3;

namespace {

struct Options {
  int days = VISS_VARIANT_10M ? 1 : 450;
  int first_day = 1;
  std::string data_dir = VISS_VARIANT_10M ? "./earth_10Mhz/" : "./earth_1Mhz/";
  std::string out_dir = VISS_VARIANT_BLOCKAGE ? (VISS_VARIANT_10M ? "3dblockage10M/" : "3dblockage/")
                                              : (VISS_VARIANT_10M ? "3dnoblockage10M/" : "3dnoblockage/");
  bool fp64 = false;
  // the blockage program's DCF (vissgen3d_blockage.cu:133-139): shell k gets
  // shell k+1's density, dcf[k] = the un-shifted dcf[k+1] for 1 <= k < nr;
  // its dcf[nr] reads past the reference's arrays and stays un-shifted here
  bool ref_dcf_shift = false;
  int max_devices = VISS_VARIANT_10M ? 1 : 1 << 20;
};

std::mutex g_io;  // the reference's omp critical sections

[[noreturn]] void die(const std::string &where, int status) {
  char buf[512];
  viss_last_error(buf, sizeof(buf));
  std::fprintf(stderr, "%s failed: %s (%d): %s\n", where.c_str(), viss_status_string(status), status, buf);
  std::exit(1);
}

#define VCALL(expr)                    \
  do {                                 \
    int st_ = (expr);                  \
    if (st_ != VISS_OK) die(#expr, st_); \
  } while (0)

#define CUCALL(expr)                                                                   \
  do {                                                                                 \
    cudaError_t e_ = (expr);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      std::fprintf(stderr, "CUDA Error: %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, \
                   __LINE__);                                                          \
      std::exit(1);                                                                    \
    }                                                                                  \
  } while (0)

template <class T>
T *dalloc(size_t n) {
  void *p = nullptr;
  CUCALL(cudaMalloc(&p, (n ? n : 1) * sizeof(T)));
  return static_cast<T *>(p);
}

template <class T>
T *upload(const std::vector<T> &v) {
  T *p = dalloc<T>(v.size());
  if (!v.empty()) CUCALL(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return p;
}

struct SkyInputs {
  int npix = 0;
  std::vector<float> B, theta, phi;
};

// One observation day on one device (vissgen3d_blockage.cu:279-556).
void run_day(int p, const Options &opt, const SkyInputs &sky, int nr, double thr,
             float s_pix) {
  const int npix = sky.npix;
  std::vector<float> cu, cv, cw, a1, b1, c1, a2, b2, c2, cbll;
  long uvw_index, xyz1_index, xyz2_index, bll_index;
  {
    std::lock_guard<std::mutex> lock(g_io);
    const std::string day = std::to_string(p + 1) + "day1M.txt";
    std::string path = opt.data_dir + "uvw" + day;
    std::cout << "address_uvw: " << path << std::endl;
    uvw_index = read_rows3(path, cu, cv, cw);
    std::cout << "uvw_index: " << uvw_index << std::endl;
    path = opt.data_dir + "xyza" + day;
    std::cout << "address_xyz1: " << path << std::endl;
    xyz1_index = read_rows3(path, a1, b1, c1);
    std::cout << "xyz1_index: " << xyz1_index << std::endl;
    path = opt.data_dir + "xyzb" + day;
    std::cout << "address_xyz2: " << path << std::endl;
    xyz2_index = read_rows3(path, a2, b2, c2);
    std::cout << "xyz2_index: " << xyz2_index << std::endl;
    path = opt.data_dir + "bll" + day;
    std::cout << "address_bll: " << path << std::endl;
    bll_index = read_rows1(path, cbll);
    std::cout << "bll_index: " << bll_index << std::endl;
  }
  const long amount = uvw_index / 2;  // the reference's ceil(uvw_index/2) on ints
  std::cout << "amount: " << amount << std::endl;
  if (xyz1_index < uvw_index || xyz2_index < uvw_index || bll_index < uvw_index) {
    std::fprintf(stderr, "day %d: xyza/xyzb/bll have fewer rows than uvw (%ld, %ld, %ld < %ld)\n",
                 p + 1, xyz1_index, xyz2_index, bll_index, uvw_index);
    std::exit(1);
  }
  std::vector<float> image(static_cast<size_t>(npix), 0.0f);
  std::vector<std::complex<float>> Vh(3);
  if (uvw_index > 0) {
    const long n = uvw_index;
    // per-row geometry in FP64 (the text values are FP32; the conversion is exact)
    std::vector<double> uvw(3 * n), w_off(n), P(6 * n);
    std::vector<int32_t> refs(3 * n);
    for (long i = 0; i < n; ++i) {
      uvw[3 * i] = cu[i]; uvw[3 * i + 1] = cv[i]; uvw[3 * i + 2] = cw[i];
      w_off[i] = -static_cast<double>(cw[i]);  // w(n-1) convention of the forward (:95)
      P[3 * i] = a1[i]; P[3 * i + 1] = b1[i]; P[3 * i + 2] = c1[i];
      P[3 * (n + i)] = a2[i]; P[3 * (n + i) + 1] = b2[i]; P[3 * (n + i) + 2] = c2[i];
      refs[3 * i] = static_cast<int32_t>(i);
      refs[3 * i + 1] = static_cast<int32_t>(n + i);
      refs[3 * i + 2] = -1;
    }
    std::vector<float> wv(cw.begin(), cw.begin() + n);  // all bll rows feed the histogram
    float *d_theta = upload(sky.theta), *d_phi = upload(sky.phi), *d_B = upload(sky.B);
    double *d_lmn = dalloc<double>(3 * static_cast<size_t>(npix));
    float *d_Bs = dalloc<float>(npix);
    double *d_uvw = upload(uvw), *d_off = upload(w_off), *d_P = upload(P);
    int32_t *d_refs = upload(refs);
    double *d_occ = dalloc<double>(4 * 2 * static_cast<size_t>(n));
    float *d_w = upload(wv), *d_bll = upload(cbll);
    float *d_V = dalloc<float>(2 * static_cast<size_t>(n) + 2);
    float *d_coef = dalloc<float>(2 * static_cast<size_t>(n));
    float *d_img = dalloc<float>(npix);
    int32_t *d_gs = dalloc<int32_t>(n);
    uint32_t *d_counts = dalloc<uint32_t>(nr);
    float *d_dcf = dalloc<float>(nr + 1), *d_dg = dalloc<float>(n), *d_wt = dalloc<float>(n);
    const int flags = opt.fp64 ? VISS_FP64 : 0;

    // healpix_moonback_pre (:401)
    VCALL(viss_sky_pre(npix, d_theta, d_phi, d_B, s_pix, d_lmn, d_Bs, nullptr));
    // occulter rows of both satellites of every row, the reference's fixed cone (:249-252)
    VCALL(viss_occulters(2 * n, d_P, 0.0, 1, thr, d_occ, nullptr));
    CUCALL(cudaMemset(d_V, 0, (2 * static_cast<size_t>(n) + 2) * sizeof(float)));
    std::cout << "Viss Computing... Here is gpu running process " << p + 1 << std::endl;
    if (amount > 0) {
      // healpix_moonback_viss (:417): first half, masked, w(n-1), then the mirror (:100)
      viss_plan *fplan = nullptr;
      VCALL(viss_plan_create(&fplan));
      VCALL(viss_plan_set_pixels(fplan, npix, d_lmn, nullptr));
      VCALL(viss_plan_set_samples(fplan, amount, d_uvw, d_off, d_refs, 2 * n, d_occ, nullptr));
      VCALL(viss_forward(fplan, d_Bs, d_V, flags, nullptr));
      VCALL(viss_plan_last_counts(fplan, nullptr, nullptr));   // a bounded wait that gave up
      VCALL(viss_conj_mirror(amount, d_V, nullptr));
      VCALL(viss_plan_destroy(fplan));
    }
    CUCALL(cudaMemcpy(Vh.data(), d_V, sizeof(float) * 2 * std::min<long>(3, n), cudaMemcpyDeviceToHost));
    std::cout << "Period " << p + 1 << " Viss Computing Success!" << std::endl;
    for (int i = 0; i <= 2 && i < n; ++i)
      std::cout << "Viss[" << i << "]: (" << Vh[i].real() << "," << Vh[i].imag() << ")" << std::endl;
    // shells + DCF (:447-486), un-shifted formula
    VCALL(viss_dcf(bll_index, d_bll, nr, 1, d_gs, d_counts, d_dcf, nullptr));
    if (opt.ref_dcf_shift && nr > 1) {
      float *d_tmp = nullptr;
      CUCALL(cudaMalloc(&d_tmp, sizeof(float) * (nr - 1)));
      CUCALL(cudaMemcpy(d_tmp, d_dcf + 2, sizeof(float) * (nr - 1), cudaMemcpyDeviceToDevice));
      CUCALL(cudaMemcpy(d_dcf + 1, d_tmp, sizeof(float) * (nr - 1), cudaMemcpyDeviceToDevice));
      CUCALL(cudaFree(d_tmp));
    }
    std::cout << "Period " << p + 1 << " calculateDcf..." << std::endl;
    // viss_gamma_trans (:494): w-rotation of every row, dg, and the clamped weights (:178,187)
    VCALL(viss_wrot(n, d_w, d_V, nullptr));
    VCALL(viss_weights(n, d_w, d_bll, d_gs, d_dcf, nr, d_dg, d_wt, nullptr));
    std::cout << "Period " << p + 1 << " viss and gamma..." << std::endl;
    // computeC (:507) over every row, phase u l + v m + w n
    VCALL(viss_scale_coef(n, d_wt, d_V, d_coef, nullptr));
    viss_plan *iplan = nullptr;
    VCALL(viss_plan_create(&iplan));
    VCALL(viss_plan_set_pixels(iplan, npix, d_lmn, nullptr));
    VCALL(viss_plan_set_samples(iplan, n, d_uvw, nullptr, VISS_VARIANT_BLOCKAGE ? d_refs : nullptr,
                                VISS_VARIANT_BLOCKAGE ? 2 * n : 0, VISS_VARIANT_BLOCKAGE ? d_occ : nullptr,
                                nullptr));
    VCALL(viss_adjoint(iplan, d_coef, d_img, 1.0f, flags, nullptr));
    VCALL(viss_plan_last_counts(iplan, nullptr, nullptr));
    VCALL(viss_plan_destroy(iplan));
    CUCALL(cudaMemcpy(image.data(), d_img, sizeof(float) * npix, cudaMemcpyDeviceToHost));
    std::cout << "Period " << p + 1 << " compute C success" << std::endl;
    void *bufs[] = {d_theta, d_phi, d_B, d_lmn, d_Bs, d_uvw, d_off, d_P, d_refs, d_occ, d_w, d_bll,
                    d_V, d_coef, d_img, d_gs, d_counts, d_dcf, d_dg, d_wt};
    for (void *b : bufs) cudaFree(b);
  }
  for (int i = 0; i <= 2 && i < npix; ++i) std::cout << "C[" << i << "]: (" << image[i] << ",0)" << std::endl;
  {
    std::lock_guard<std::mutex> lock(g_io);
    const std::string path = opt.out_dir + "C" + std::to_string(p + 1) + "day1M.txt";
    std::cout << "Period " << p + 1 << " save address_C: " << path << std::endl;
    if (!viss_host::write_column(path, image))
      std::fprintf(stderr, "could not write %s (does the directory exist?)\n", path.c_str());
    std::cout << "Period " << p + 1 << " save C success!" << std::endl;
  }
}

int vissGen(float frequency, const Options &opt) {
  const auto t0 = std::chrono::steady_clock::now();
  int nDevices = 0;
  CUCALL(cudaGetDeviceCount(&nDevices));
  nDevices = std::max(1, std::min(nDevices, opt.max_devices));
  std::cout << "devices: " << nDevices << std::endl;
  std::cout << "frequency: " << frequency << std::endl;
  std::cout << "days: " << opt.days << std::endl;

  SkyInputs sky;
  {
    const std::string suffix = VISS_VARIANT_10M ? "_10Mhz.txt" : ".txt";
    viss_host::TokenReader Bf(opt.data_dir + "B" + suffix);
    viss_host::TokenReader tf(opt.data_dir + "theta_heal" + suffix);
    viss_host::TokenReader pf(opt.data_dir + "phi_heal" + suffix);
    if (!Bf.next_int(sky.npix) || sky.npix <= 0) {
      std::fprintf(stderr, "cannot read npix from %sB%s\n", opt.data_dir.c_str(), suffix.c_str());
      return 1;
    }
    std::cout << "npix: " << sky.npix << std::endl;
    sky.B.resize(sky.npix); sky.theta.resize(sky.npix); sky.phi.resize(sky.npix);
    for (int i = 0; i < sky.npix; ++i) {
      if (!(Bf.next(sky.B[i]) && tf.next(sky.theta[i]) && pf.next(sky.phi[i]))) {
        std::fprintf(stderr, "B/theta/phi files have fewer than npix = %d values\n", sky.npix);
        return 1;
      }
    }
  }
  std::cout << "load B.txt, theta_heal.txt, phi_heal.txt in CPU success" << std::endl;

  const int nside = static_cast<int>(std::round(std::sqrt(sky.npix / 12)));
  const float s = 4 * M_PI / sky.npix;                 // :242 (FP32 as stored there)
  const float res = std::sqrt(4 * M_PI / sky.npix);
  const float R = 1737.1e3f, h = 300e3f;               // :249-252
  const float theta = std::asin(R / (R + h));
  const float phi = M_PI - theta;
  std::cout << "theta: " << theta << std::endl;
  std::cout << "phi: " << phi << std::endl;
  const float bl_max = 100e3f;                         // :257-259
  const float lamda = 3e8 / frequency;
  const float nr_f = std::ceil(bl_max / lamda * 2);
  const int nr = static_cast<int>(nr_f);
  std::cout << "nside: " << nside << std::endl;
  std::cout << "s: " << s << std::endl;
  std::cout << "res: " << res << std::endl;
  std::cout << "theta: " << theta << std::endl;
  std::cout << "lamda: " << lamda << std::endl;
  std::cout << "nr: " << nr_f << std::endl;
  const double thr = viss_cone_threshold(R, h);

  std::vector<std::thread> threads;
  for (int tid = 0; tid < nDevices; ++tid) {
    threads.emplace_back([&, tid] {
      CUCALL(cudaSetDevice(tid));
      {
        std::lock_guard<std::mutex> lock(g_io);
        std::cout << "Thread " << tid << " is running on device " << tid << std::endl;
      }
      for (int p = opt.first_day - 1 + tid; p < opt.first_day - 1 + opt.days; p += nDevices) {
        {
          std::lock_guard<std::mutex> lock(g_io);
          std::cout << "for loop: " << p + 1 << std::endl;
        }
        run_day(p, opt, sky, nr, thr, s);
      }
    });
  }
  for (auto &t : threads) t.join();
  const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout << "total time: " << total << "s" << std::endl;
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  Options opt;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&](const char *name) -> std::string {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "%s needs a value\n", name);
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--days") opt.days = std::atoi(val("--days").c_str());
    else if (a == "--first-day") opt.first_day = std::atoi(val("--first-day").c_str());
    else if (a == "--data-dir") opt.data_dir = val("--data-dir");
    else if (a == "--out-dir") opt.out_dir = val("--out-dir");
    else if (a == "--fp64") opt.fp64 = true;
    else if (a == "--ref-dcf-shift") opt.ref_dcf_shift = true;
    else if (a == "--devices") opt.max_devices = std::atoi(val("--devices").c_str());
    else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  if (!opt.data_dir.empty() && opt.data_dir.back() != '/') opt.data_dir += '/';
  if (!opt.out_dir.empty() && opt.out_dir.back() != '/') opt.out_dir += '/';
  return vissGen(VISS_VARIANT_10M ? 1e7f : 1e6f, opt);
}
