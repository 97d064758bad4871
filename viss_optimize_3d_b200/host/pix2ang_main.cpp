// pix2ang_main.cpp -- drop-in replacement for the reference executable
// pix2ang (pix2ang.cu:163-276): reads B.txt from the working directory
// (npix, then npix values), derives nside = round(sqrt(npix/12)) and writes
// the NESTED pixel-centre colatitudes and longitudes to theta_heal.txt and
// phi_heal.txt, one value per line.  The tables come from viss_pix2ang, which
// follows the HEALPix definition (the reference kernel f_pix2and_nest,
// pix2ang.cu:92-160, indexes its tables 1-based and produces no valid
// centre).  Optional flags: --ring (RING order instead of NESTED),
// --in PATH (default B.txt), --out-dir PATH (default .).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "textio.h"
#include "viss.h"

int main(int argc, char **argv) {
  int scheme = VISS_NESTED;
  std::string in = "B.txt", out_dir = ".";
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    if (a == "--ring") scheme = VISS_RING;
    else if (a == "--in" && i + 1 < argc) in = argv[++i];
    else if (a == "--out-dir" && i + 1 < argc) out_dir = argv[++i];
    else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return 2;
    }
  }
  viss_host::TokenReader B(in);
  int npix = 0;
  if (!B.next_int(npix) || npix <= 0) {
    std::fprintf(stderr, "cannot read npix from %s\n", in.c_str());
    return 1;
  }
  std::cout << "npix: " << npix << std::endl;
  const int nside = static_cast<int>(std::round(std::sqrt(npix / 12)));
  if (12LL * nside * nside != npix) {
    std::fprintf(stderr, "npix = %d is not 12 nside^2\n", npix);
    return 1;
  }
  const float s = 4 * M_PI / npix;
  const float res = std::sqrt(4 * M_PI / npix);
  std::cout << "res: " << res << std::endl;
  std::cout << "s: " << s << std::endl;
  std::cout << "nside: " << nside << std::endl;
  std::cout << "npface: " << nside * nside << std::endl;
  std::cout << "nl4: " << 4 * nside << std::endl;
  std::cout << "fact1: " << 1.0f / (3.0f * nside * nside) << std::endl;
  std::cout << "fact2: " << 2.0f / (3.0f * nside) << std::endl;

  double *d_theta = nullptr, *d_phi = nullptr;
  if (cudaMalloc(&d_theta, sizeof(double) * npix) != cudaSuccess ||
      cudaMalloc(&d_phi, sizeof(double) * npix) != cudaSuccess) {
    std::fprintf(stderr, "cudaMalloc failed\n");
    return 1;
  }
  const int st = viss_pix2ang(nside, scheme, 0, npix, d_theta, d_phi, nullptr, nullptr);
  if (st != VISS_OK) {
    char buf[512];
    viss_last_error(buf, sizeof(buf));
    std::fprintf(stderr, "viss_pix2ang failed: %s\n", buf);
    return 1;
  }
  std::vector<double> th(npix), ph(npix);
  cudaMemcpy(th.data(), d_theta, sizeof(double) * npix, cudaMemcpyDeviceToHost);
  cudaMemcpy(ph.data(), d_phi, sizeof(double) * npix, cudaMemcpyDeviceToHost);
  cudaFree(d_theta);
  cudaFree(d_phi);
  // the reference writes FP32 values (pix2ang.cu:42-58)
  std::vector<float> tf(th.begin(), th.end()), pf(ph.begin(), ph.end());
  const bool ok = viss_host::write_column(out_dir + "/theta_heal.txt", tf) &&
                  viss_host::write_column(out_dir + "/phi_heal.txt", pf);
  if (!ok) {
    std::fprintf(stderr, "could not write theta_heal.txt / phi_heal.txt in %s\n", out_dir.c_str());
    return 1;
  }
  return 0;
}
