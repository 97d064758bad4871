// vissgen_stream_main.cpp -- the reference's multi-day loop (vissGen,
// vissgen3d_blockage.cu:195-563) as a streaming pipeline over binary day
// files (host/dayfile.h), with the day sum of its notebooks
// (healpix3d_blockage.ipynb:103-116) kept on the device.
//
// Per GPU (days round-robin over GPUs, one host thread each, as the
// reference's OpenMP loop, :271-279):
//   * the sky, its (l, m, n) records and both plans' pixel staging are set up
//     once, not once per day (the reference re-uploads and re-derives them
//     every day, :281-306, :401);
//   * a loader thread reads day d+1 straight into pinned host memory and
//     copies it to the device on a copy stream while day d computes (two
//     slots, ordered by CUDA events);
//   * the per-row geometry the reference builds in host loops is built by
//     one device kernel (viss_stage_day_rows);
//   * each day's image is summed on the device in FP64, non-finite pixels
//     as 0 (viss_accumulate_image); per-day images are written by a writer
//     thread from pinned memory when asked for.
// After the last day the per-GPU FP64 sums are reduced onto GPU 0 by one NCCL
// reduce (SUM), over NVLink where the GPUs have it; only that sum is copied
// to the host (one GPU: a plain copy, or the NCCL path with --nccl-reduce).
// The arithmetic per day is that of the drop-in executables
// (host/vissgen_main.cpp): occultation rows of both satellites with the
// reference's fixed cone, forward of the unique half with off = -w, conjugate
// mirror, shells + DCF over every row, w-rotation, weights, imaging over
// every row (occulted with --blockage 1).  With --fold-mirrors (rows checked
// on the host to be exact mirrors) imaging and DCF run over the unique half
// with multiplicity 2 and scale 2: the same sum with a third less work.
//
//   vissgen_stream --sky SKY.vsky --days-dir DIR [--first-day D] [--days N]
//                  [--frequency HZ] [--blockage 0|1] [--fold-mirrors] [--fp64]
//                  [--out-dir DIR [--resume]] [--sum-out FILE] [--devices N] [--nccl-reduce]
//                  [--gridded]
// --gridded images each day with viss_adjoint_gridded (per-facet NUFFTs, the
// occulted ones as a hybrid with the direct kernel; split precision): faster
// where the sky is fine against the baselines (1 MHz on Nside 512), and an
// error where no facet size keeps the grid under its limit.
// --resume skips the days whose image an earlier run already wrote to
// --out-dir (a valid C{d}.vimg) and adds those images to the day sum instead,
// so an interrupted run continues where it stopped.  Each day is one NVTX
// range ("day d") for profilers.
//   vissgen_stream --convert-text SRC --to DST [--text-10m] [--first-day D] [--days N]
//   vissgen_stream --info FILE
// Prints one JSON line with the timings at the end of a run.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nccl.h>
#include <nvtx3/nvToolsExt.h>

#include "dayfile.h"
#include "textio.h"
#include "viss.h"

namespace {

using viss_host::FileHeader;

struct Options {
  std::string sky, days_dir, out_dir, sum_out;
  int first_day = 1, days = 1, max_devices = 1 << 20;
  double frequency = 1e6;
  bool blockage = true, fold = false, fp64 = false, resume = false;
  bool nccl_reduce = false;   // --nccl-reduce: the NCCL reduce even on one GPU
  bool gridded = false;       // --gridded: viss_adjoint_gridded for imaging
  std::string convert_src, convert_dst, info;
  bool text_10m = false;
};

[[noreturn]] void die(const std::string &msg) {
  std::fprintf(stderr, "vissgen_stream: %s\n", msg.c_str());
  std::exit(1);
}

void vcall(int st, const char *what) {
  if (st == VISS_OK) return;
  char buf[512];
  viss_last_error(buf, sizeof(buf));
  die(std::string(what) + ": " + viss_status_string(st) + ": " + buf);
}

void cucall(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device buffer that grows (never shrinks) to hold n elements.
template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t cap = 0;
  void ensure(size_t n) {
    if (n <= cap && p) return;
    if (p) cucall(cudaFree(p), "cudaFree");
    cucall(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    cap = n;
  }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

struct Sky {
  int64_t npix = 0;
  std::vector<float> B, theta, phi;
};

Sky read_sky(const std::string &path) {
  FileHeader h;
  std::string err;
  std::FILE *f = viss_host::open_checked(path, "VISSSKY", viss_host::kSkyFloatsPerPixel, h, err);
  if (!f) die(err);
  if (h.elem_bytes != 4 || h.count <= 0) die(path + ": expected float32 pixels");
  Sky s;
  s.npix = h.count;
  s.B.resize(h.count);
  s.theta.resize(h.count);
  s.phi.resize(h.count);
  const bool ok = std::fread(s.B.data(), 4, h.count, f) == static_cast<size_t>(h.count) &&
                  std::fread(s.theta.data(), 4, h.count, f) == static_cast<size_t>(h.count) &&
                  std::fread(s.phi.data(), 4, h.count, f) == static_cast<size_t>(h.count);
  std::fclose(f);
  if (!ok) die(path + ": short read");
  return s;
}

std::string day_file(const Options &o, int day) {
  return o.days_dir + "day" + std::to_string(day) + ".vday";
}

// Exact mirrors: row i + n/2 is row i with u -> -u and the same positions and bll.
bool rows_are_mirrors(const float *rows, int64_t n) {
  if (n % 2) return false;
  const int64_t m = n / 2;
  const float *uvw = rows, *xa = rows + 3 * n, *xb = rows + 6 * n, *bll = rows + 9 * n;
  for (int64_t i = 0; i < m; ++i) {
    for (int c = 0; c < 3; ++c) {
      if (uvw[3 * (m + i) + c] != -uvw[3 * i + c] || xa[3 * (m + i) + c] != xa[3 * i + c] ||
          xb[3 * (m + i) + c] != xb[3 * i + c])
        return false;
    }
    if (bll[m + i] != bll[i]) return false;
  }
  return true;
}

// ---------------------------------------------------------------- pipeline
struct Slot {
  float *host = nullptr;   // pinned: the day file's payload
  size_t host_cap = 0;     // floats
  DevBuf<float> dev;       // the same on the device
  cudaEvent_t copied{}, consumed{};
  int64_t n = 0;
  int day = 0;
  bool loaded = false, failed = false;
  std::string error;
};

struct DayTiming {
  int day;
  int64_t rows;
  double gpu_ms;
};

class DevicePipeline {
 public:
  DevicePipeline(int dev, const Options &o, const Sky &sky, std::vector<int> days)
      : dev_(dev), o_(o), sky_(sky), days_(std::move(days)) {}

  // The day sum on this pipeline's device (FP64, npix), valid after run().
  double *device_sum() const { return sum_.p; }
  int device() const { return dev_; }

  void run(std::vector<DayTiming> &timings) {
    cucall(cudaSetDevice(dev_), "cudaSetDevice");
    cucall(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking), "stream");
    cucall(cudaStreamCreateWithFlags(&xs_, cudaStreamNonBlocking), "stream");
    for (Slot &s : slots_) {
      cucall(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming), "event");
      cucall(cudaEventCreateWithFlags(&s.consumed, cudaEventDisableTiming), "event");
    }
    setup_sky();
    std::thread loader([this] { load_loop(); });
    std::thread writer;
    if (!o_.out_dir.empty()) writer = std::thread([this] { write_loop(); });
    cudaEvent_t e0, e1;
    cucall(cudaEventCreate(&e0), "event");
    cucall(cudaEventCreate(&e1), "event");
    for (size_t k = 0; k < days_.size(); ++k) {
      Slot &s = slots_[k % 2];
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return s.loaded; });
        if (s.failed) {
          abort_ = true;
          cv_.notify_all();
          lk.unlock();
          loader.join();
          die(s.error);
        }
      }
      // the slot's fields belong to the loader again once `loaded` is cleared
      const int64_t n = s.n;
      const int day = s.day;
      nvtxRangePushA(("day " + std::to_string(day)).c_str());
      cucall(cudaEventRecord(e0, cs_), "event");
      ensure_rows(n);
      cucall(cudaStreamWaitEvent(cs_, s.copied, 0), "wait");
      if (n > 0) {
        const float *d = s.dev.p;
        vcall(viss_stage_day_rows(n, d, d + 3 * n, d + 6 * n, uvw_.p, off_.p, P_.p, refs_.p, w_.p,
                                  cs_),
              "viss_stage_day_rows");
        cucall(cudaMemcpyAsync(bll_.p, d + 9 * n, n * sizeof(float), cudaMemcpyDeviceToDevice, cs_),
               "bll");
      }
      cucall(cudaEventRecord(s.consumed, cs_), "event");
      {
        std::lock_guard<std::mutex> lk(mu_);
        s.loaded = false;
      }
      cv_.notify_all();
      compute_day(n);
      if (!o_.out_dir.empty()) queue_image(day);
      vcall(viss_accumulate_image(sky_.npix, img_.p, sum_.p, cs_), "viss_accumulate_image");
      cucall(cudaEventRecord(e1, cs_), "event");
      cucall(cudaEventSynchronize(e1), "sync");
      float ms = 0;
      cucall(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
      nvtxRangePop();
      timings.push_back({day, n, ms});
    }
    loader.join();
    {
      std::lock_guard<std::mutex> lk(mu_);
      writer_done_ = true;
    }
    cv_.notify_all();
    if (writer.joinable()) writer.join();
    if (!write_error_.empty()) die(write_error_);
    cucall(cudaStreamSynchronize(cs_), "sync");
    vcall(viss_plan_destroy(fplan_), "viss_plan_destroy");
    vcall(viss_plan_destroy(iplan_), "viss_plan_destroy");
    for (Slot &s : slots_) {
      if (s.host) cudaFreeHost(s.host);
      cudaEventDestroy(s.copied);
      cudaEventDestroy(s.consumed);
    }
    for (auto &h : img_host_)
      if (h) cudaFreeHost(h);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(cs_);
    cudaStreamDestroy(xs_);
  }

 private:
  void setup_sky() {
    const int64_t npix = sky_.npix;
    DevBuf<float> th, ph, B;
    th.ensure(npix);
    ph.ensure(npix);
    B.ensure(npix);
    cucall(cudaMemcpy(th.p, sky_.theta.data(), npix * 4, cudaMemcpyHostToDevice), "sky");
    cucall(cudaMemcpy(ph.p, sky_.phi.data(), npix * 4, cudaMemcpyHostToDevice), "sky");
    cucall(cudaMemcpy(B.p, sky_.B.data(), npix * 4, cudaMemcpyHostToDevice), "sky");
    lmn_.ensure(3 * npix);
    Bs_.ensure(npix);
    img_.ensure(npix);
    sum_.ensure(npix);
    const float s = 4 * M_PI / npix;  // vissgen3d_blockage.cu:242 (FP32)
    vcall(viss_sky_pre(npix, th.p, ph.p, B.p, s, lmn_.p, Bs_.p, cs_), "viss_sky_pre");
    cucall(cudaMemsetAsync(sum_.p, 0, npix * sizeof(double), cs_), "memset");
    vcall(viss_plan_create(&fplan_), "viss_plan_create");
    vcall(viss_plan_create(&iplan_), "viss_plan_create");
    vcall(viss_plan_set_pixels(fplan_, npix, lmn_.p, cs_), "viss_plan_set_pixels");
    vcall(viss_plan_set_pixels(iplan_, npix, lmn_.p, cs_), "viss_plan_set_pixels");
    cucall(cudaStreamSynchronize(cs_), "sync");
    // the reference's constants (vissgen3d_blockage.cu:249-259)
    const float R = 1737.1e3f, h = 300e3f;
    thr_ = viss_cone_threshold(R, h);
    const float lamda = static_cast<float>(3e8 / o_.frequency);
    nr_ = static_cast<int>(std::ceil(100e3f / lamda * 2));
    counts_.ensure(nr_);
    dcf_.ensure(nr_ + 1);
  }

  void ensure_rows(int64_t n) {
    uvw_.ensure(3 * n);
    off_.ensure(n);
    P_.ensure(6 * n);
    refs_.ensure(3 * n);
    w_.ensure(n);
    bll_.ensure(n);
    occ_.ensure(8 * n);
    V_.ensure(2 * n + 2);
    coef_.ensure(2 * n);
    gs_.ensure(n);
    dg_.ensure(n);
    wt_.ensure(n);
  }

  void compute_day(int64_t n) {
    const int flags = o_.fp64 ? VISS_FP64 : 0;
    const int64_t amount = n / 2;
    vcall(viss_occulters(2 * n, P_.p, 0.0, 1, thr_, occ_.p, cs_), "viss_occulters");
    cucall(cudaMemsetAsync(V_.p, 0, (2 * n + 2) * sizeof(float), cs_), "memset");
    if (amount > 0) {
      vcall(viss_plan_set_samples(fplan_, amount, uvw_.p, off_.p, refs_.p, 2 * n, occ_.p, cs_),
            "viss_plan_set_samples");
      vcall(viss_forward(fplan_, Bs_.p, V_.p, flags, cs_), "viss_forward");
      vcall(viss_conj_mirror(amount, V_.p, cs_), "viss_conj_mirror");
    }
    // rows that take part in the shells, the weights and imaging: all of
    // them, or the unique half counted twice (--fold-mirrors)
    const int64_t m = o_.fold ? amount : n;
    const int mult = o_.fold ? 2 : 1;
    const float scale = o_.fold ? 2.0f : 1.0f;
    vcall(viss_dcf(m, bll_.p, nr_, mult, gs_.p, counts_.p, dcf_.p, cs_), "viss_dcf");
    vcall(viss_wrot(m, w_.p, V_.p, cs_), "viss_wrot");
    vcall(viss_weights(m, w_.p, bll_.p, gs_.p, dcf_.p, nr_, dg_.p, wt_.p, cs_), "viss_weights");
    vcall(viss_scale_coef(m, wt_.p, V_.p, coef_.p, cs_), "viss_scale_coef");
    if (m > 0) {
      vcall(viss_plan_set_samples(iplan_, m, uvw_.p, nullptr, o_.blockage ? refs_.p : nullptr,
                                  o_.blockage ? 2 * n : 0, o_.blockage ? occ_.p : nullptr, cs_),
            "viss_plan_set_samples");
      // set_samples synchronised cs_, so the forward has finished: did any of
      // its bounded waits give up?
      if (amount > 0) vcall(viss_plan_last_counts(fplan_, nullptr, nullptr), "viss_forward");
      if (o_.gridded) {
        vcall(viss_adjoint_gridded(iplan_, coef_.p, img_.p, scale, 0, 0, cs_), "viss_adjoint_gridded");
        // the occulted one ran the direct kernel for the pairs it did not grid
        if (o_.blockage) vcall(viss_plan_last_counts(iplan_, nullptr, nullptr), "viss_adjoint_gridded");
      } else {
        vcall(viss_adjoint(iplan_, coef_.p, img_.p, scale, flags, cs_), "viss_adjoint");
        vcall(viss_plan_last_counts(iplan_, nullptr, nullptr), "viss_adjoint");
      }
    } else {
      cucall(cudaMemsetAsync(img_.p, 0, sky_.npix * sizeof(float), cs_), "memset");
    }
  }

  // loader thread: file -> pinned slot -> device slot (copy stream)
  void load_loop() {
    cucall(cudaSetDevice(dev_), "cudaSetDevice");
    for (size_t k = 0; k < days_.size(); ++k) {
      Slot &s = slots_[k % 2];
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !s.loaded || abort_; });
        if (abort_) return;
      }
      // the previous H2D from this slot has finished with the host buffer
      cucall(cudaEventSynchronize(s.copied), "sync");
      const int day = days_[k];
      const std::string path = day_file(o_, day);
      FileHeader h;
      std::string err;
      std::FILE *f = viss_host::open_checked(path, "VISSDAY", viss_host::kDayFloatsPerRow, h, err);
      bool ok = f != nullptr;
      if (ok && h.elem_bytes != 4) {
        err = path + ": expected float32 rows";
        ok = false;
      }
      const int64_t n = ok ? h.count : 0;
      const size_t floats = static_cast<size_t>(n) * viss_host::kDayFloatsPerRow;
      if (ok && floats > s.host_cap) {
        if (s.host) cucall(cudaFreeHost(s.host), "cudaFreeHost");
        cucall(cudaHostAlloc(reinterpret_cast<void **>(&s.host), floats * sizeof(float),
                             cudaHostAllocDefault),
               "cudaHostAlloc");
        s.host_cap = floats;
      }
      if (ok && floats && std::fread(s.host, sizeof(float), floats, f) != floats) {
        err = path + ": short read";
        ok = false;
      }
      if (f) std::fclose(f);
      if (ok && o_.fold && !rows_are_mirrors(s.host, n)) {
        err = path + ": --fold-mirrors needs rows n/2.. to be the exact mirrors of rows 0..n/2";
        ok = false;
      }
      if (ok && floats) {
        // the device slot is free once the compute stream has staged it
        cucall(cudaStreamWaitEvent(xs_, s.consumed, 0), "wait");
        if (floats > s.dev.cap) {
          cucall(cudaStreamSynchronize(xs_), "sync");
          s.dev.ensure(floats);
        }
        cucall(cudaMemcpyAsync(s.dev.p, s.host, floats * sizeof(float), cudaMemcpyHostToDevice, xs_),
               "H2D");
      }
      cucall(cudaEventRecord(s.copied, xs_), "event");
      {
        std::lock_guard<std::mutex> lk(mu_);
        s.n = n;
        s.day = day;
        s.failed = !ok;
        s.error = err;
        s.loaded = true;
      }
      cv_.notify_all();
      if (!ok) return;
    }
  }

  // per-day image: device -> pinned (compute stream) -> file (writer thread)
  void queue_image(int day) {
    const int b = static_cast<int>(queued_ % 2);
    {
      std::unique_lock<std::mutex> lk(mu_);
      cv_.wait(lk, [&] { return written_ + 2 > queued_; });  // buffer b written out
    }
    if (!img_host_[b])
      cucall(cudaHostAlloc(reinterpret_cast<void **>(&img_host_[b]), sky_.npix * sizeof(float),
                           cudaHostAllocDefault),
             "cudaHostAlloc");
    if (!img_ev_[b]) cucall(cudaEventCreateWithFlags(&img_ev_[b], cudaEventDisableTiming), "event");
    cucall(cudaMemcpyAsync(img_host_[b], img_.p, sky_.npix * sizeof(float), cudaMemcpyDeviceToHost, cs_),
           "D2H");
    cucall(cudaEventRecord(img_ev_[b], cs_), "event");
    {
      std::lock_guard<std::mutex> lk(mu_);
      pending_.push_back({day, b});
      ++queued_;
    }
    cv_.notify_all();
  }

  void write_loop() {
    cucall(cudaSetDevice(dev_), "cudaSetDevice");
    for (;;) {
      std::pair<int, int> job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !pending_.empty() || writer_done_; });
        if (pending_.empty()) return;
        job = pending_.front();
        pending_.pop_front();
      }
      cucall(cudaEventSynchronize(img_ev_[job.second]), "sync");
      const FileHeader h = viss_host::make_header("VISSIMG", 4, sky_.npix, job.first, o_.frequency, 1);
      const std::string path = o_.out_dir + "C" + std::to_string(job.first) + ".vimg";
      if (!viss_host::write_file(path, h, img_host_[job.second], sky_.npix * sizeof(float))) {
        std::lock_guard<std::mutex> lk(mu_);
        if (write_error_.empty()) write_error_ = "could not write " + path;
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        ++written_;
      }
      cv_.notify_all();
    }
  }

  int dev_;
  const Options &o_;
  const Sky &sky_;
  std::vector<int> days_;
  cudaStream_t cs_{}, xs_{};
  Slot slots_[2];
  std::mutex mu_;
  std::condition_variable cv_;
  bool abort_ = false, writer_done_ = false;
  std::deque<std::pair<int, int>> pending_;
  long long queued_ = 0, written_ = 0;
  std::string write_error_;
  float *img_host_[2] = {nullptr, nullptr};
  cudaEvent_t img_ev_[2] = {nullptr, nullptr};
  viss_plan *fplan_ = nullptr, *iplan_ = nullptr;
  double thr_ = 0;
  int nr_ = 0;
  DevBuf<double> lmn_, uvw_, off_, P_, occ_, sum_;
  DevBuf<float> Bs_, img_, w_, bll_, V_, coef_, dcf_, dg_, wt_;
  DevBuf<int32_t> refs_, gs_;
  DevBuf<uint32_t> counts_;
};

// A day image written by an earlier run, if `path` holds a valid one.
bool read_day_image(const std::string &path, int64_t npix, std::vector<float> &img) {
  FileHeader h;
  std::string err;
  std::FILE *f = viss_host::open_checked(path, "VISSIMG", 1, h, err);
  if (!f) return false;
  bool ok = h.elem_bytes == 4 && h.count == npix && h.days == 1;
  if (ok) {
    img.resize(npix);
    ok = std::fread(img.data(), sizeof(float), npix, f) == static_cast<size_t>(npix);
  }
  std::fclose(f);
  return ok;
}

void nccall(ncclResult_t r, const char *what) {
  if (r != ncclSuccess) die(std::string(what) + ": " + ncclGetErrorString(r));
}

// The day sums of all pipelines' GPUs, reduced onto the first by one NCCL
// reduce (FP64 SUM), then added to `total` on the host.  With one GPU the
// reduce is skipped (communicator set-up costs about a second) unless
// `use_nccl` asks for it (a one-rank communicator; the tests use it).
void reduce_day_sums(const std::vector<std::unique_ptr<DevicePipeline>> &pipes, int64_t npix,
                     std::vector<double> &total, bool use_nccl) {
  const int n = static_cast<int>(pipes.size());
  std::vector<int> devs(n);
  for (int d = 0; d < n; ++d) devs[d] = pipes[d]->device();
  if (n == 1 && !use_nccl) {
    std::vector<double> sum(npix);
    cucall(cudaSetDevice(devs[0]), "cudaSetDevice");
    cucall(cudaMemcpy(sum.data(), pipes[0]->device_sum(), npix * sizeof(double), cudaMemcpyDeviceToHost),
           "sum");
    for (int64_t j = 0; j < npix; ++j) total[j] += sum[j];
    return;
  }
  std::vector<ncclComm_t> comms(n);
  nccall(ncclCommInitAll(comms.data(), n, devs.data()), "ncclCommInitAll");
  std::vector<cudaStream_t> st(n);
  for (int d = 0; d < n; ++d) {
    cucall(cudaSetDevice(devs[d]), "cudaSetDevice");
    cucall(cudaStreamCreateWithFlags(&st[d], cudaStreamNonBlocking), "stream");
  }
  nccall(ncclGroupStart(), "ncclGroupStart");
  for (int d = 0; d < n; ++d)
    nccall(ncclReduce(pipes[d]->device_sum(), pipes[d]->device_sum(), static_cast<size_t>(npix),
                      ncclFloat64, ncclSum, 0, comms[d], st[d]),
           "ncclReduce");
  nccall(ncclGroupEnd(), "ncclGroupEnd");
  for (int d = 0; d < n; ++d) {
    cucall(cudaSetDevice(devs[d]), "cudaSetDevice");
    cucall(cudaStreamSynchronize(st[d]), "sync");
  }
  std::vector<double> sum(npix);
  cucall(cudaSetDevice(devs[0]), "cudaSetDevice");
  cucall(cudaMemcpy(sum.data(), pipes[0]->device_sum(), npix * sizeof(double), cudaMemcpyDeviceToHost),
         "sum");
  for (int64_t j = 0; j < npix; ++j) total[j] += sum[j];
  for (int d = 0; d < n; ++d) {
    ncclCommDestroy(comms[d]);
    cudaStreamDestroy(st[d]);
  }
}

int stream(const Options &o) {
  const auto t0 = std::chrono::steady_clock::now();
  const Sky sky = read_sky(o.sky);
  // days an earlier run finished (--resume): their images go straight into the sum
  std::vector<double> total(sky.npix, 0.0);
  std::vector<int> todo;
  int resumed = 0;
  for (int k = 0; k < o.days; ++k) {
    const int day = o.first_day + k;
    std::vector<float> img;
    if (o.resume && read_day_image(o.out_dir + "C" + std::to_string(day) + ".vimg", sky.npix, img)) {
      for (int64_t j = 0; j < sky.npix; ++j) total[j] += std::isfinite(img[j]) ? img[j] : 0.0;
      ++resumed;
      continue;
    }
    todo.push_back(day);
  }
  int ndev = 0;
  if (!todo.empty()) cucall(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  ndev = std::max(1, std::min(ndev, std::min(o.max_devices, static_cast<int>(todo.size()))));
  std::vector<std::vector<int>> mine(ndev);
  for (size_t k = 0; k < todo.size(); ++k) mine[k % ndev].push_back(todo[k]);  // :279
  std::vector<std::vector<DayTiming>> timings(ndev);
  std::vector<std::unique_ptr<DevicePipeline>> pipes;
  std::vector<std::thread> threads;
  if (!todo.empty()) {
    for (int d = 0; d < ndev; ++d) pipes.emplace_back(new DevicePipeline(d, o, sky, mine[d]));
    for (int d = 0; d < ndev; ++d) threads.emplace_back([&, d] { pipes[d]->run(timings[d]); });
    for (auto &t : threads) t.join();
    reduce_day_sums(pipes, sky.npix, total, o.nccl_reduce);
  }
  // day sum: the resumed days plus the reduced device sums
  if (!o.sum_out.empty()) {
    const FileHeader h = viss_host::make_header("VISSIMG", 8, sky.npix, o.first_day, o.frequency, o.days);
    if (!viss_host::write_file(o.sum_out, h, total.data(), total.size() * sizeof(double)))
      die("could not write " + o.sum_out);
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::string per;
  double gpu_ms = 0;
  long long rows = 0;
  for (int d = 0; d < ndev; ++d)
    for (const DayTiming &t : timings[d]) {
      per += (per.empty() ? "" : ", ") + std::string("[") + std::to_string(t.day) + ", " +
             std::to_string(t.rows) + ", " + std::to_string(t.gpu_ms) + "]";
      gpu_ms += t.gpu_ms;
      rows += t.rows;
    }
  std::printf("{\"days\": %d, \"resumed_days\": %d, \"devices\": %d, \"npix\": %lld, "
              "\"rows\": %lld, \"wall_s\": %.4f, \"gpu_ms_total\": %.3f, \"per_day\": [%s]}\n",
              o.days, resumed, todo.empty() ? 0 : ndev, static_cast<long long>(sky.npix), rows, wall,
              gpu_ms, per.c_str());
  return 0;
}

// Text day files of the reference (vissgen3d_blockage.cu:216-237,309-391) -> binary.
int convert(const Options &o) {
  const std::string src = o.convert_src, dst = o.convert_dst;
  const std::string suffix = o.text_10m ? "_10Mhz.txt" : ".txt";
  viss_host::TokenReader Bf(src + "B" + suffix), tf(src + "theta_heal" + suffix),
      pf(src + "phi_heal" + suffix);
  int npix = 0;
  if (!Bf.next_int(npix) || npix <= 0) die("cannot read npix from " + src + "B" + suffix);
  std::vector<float> sky(3 * static_cast<size_t>(npix));
  for (int i = 0; i < npix; ++i)
    if (!(Bf.next(sky[i]) && tf.next(sky[npix + i]) && pf.next(sky[2 * npix + i])))
      die("B/theta/phi files have fewer than npix values");
  if (!viss_host::write_file(dst + "sky.vsky", viss_host::make_header("VISSSKY", 4, npix, 1, 0, 1),
                             sky.data(), sky.size() * 4))
    die("could not write " + dst + "sky.vsky");
  for (int day = o.first_day; day < o.first_day + o.days; ++day) {
    const std::string tag = std::to_string(day) + "day1M.txt";
    std::vector<float> a[3], b[3], c[3], bll;
    const long n = viss_host::read_rows3(src + "uvw" + tag, a[0], b[0], c[0]);
    const long n1 = viss_host::read_rows3(src + "xyza" + tag, a[1], b[1], c[1]);
    const long n2 = viss_host::read_rows3(src + "xyzb" + tag, a[2], b[2], c[2]);
    const long nb = viss_host::read_rows1(src + "bll" + tag, bll);
    if (n1 < n || n2 < n || nb < n) die("day " + std::to_string(day) + ": xyza/xyzb/bll have fewer rows than uvw");
    std::vector<float> rows(static_cast<size_t>(n) * viss_host::kDayFloatsPerRow);
    for (long i = 0; i < n; ++i)
      for (int f = 0; f < 3; ++f) {
        rows[3 * (f * n + i)] = a[f][i];
        rows[3 * (f * n + i) + 1] = b[f][i];
        rows[3 * (f * n + i) + 2] = c[f][i];
      }
    for (long i = 0; i < n; ++i) rows[9 * n + i] = bll[i];
    const std::string out = dst + "day" + std::to_string(day) + ".vday";
    if (!viss_host::write_file(out, viss_host::make_header("VISSDAY", 4, n, day, 0, 1), rows.data(),
                               rows.size() * 4))
      die("could not write " + out);
    std::printf("%s: %ld rows\n", out.c_str(), n);
  }
  return 0;
}

int info(const std::string &path) {
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) die("cannot open " + path);
  FileHeader h;
  const bool ok = std::fread(&h, sizeof(h), 1, f) == 1;
  std::fclose(f);
  if (!ok) die(path + ": no header");
  const char *magics[] = {"VISSDAY", "VISSSKY", "VISSIMG"};
  const int per[] = {viss_host::kDayFloatsPerRow, viss_host::kSkyFloatsPerPixel, 1};
  for (int k = 0; k < 3; ++k) {
    if (std::strncmp(h.magic, magics[k], 8) != 0) continue;
    std::string err;
    std::FILE *g = viss_host::open_checked(path, magics[k], per[k], h, err);
    if (!g) die(err);
    std::fclose(g);
    std::printf("{\"kind\": \"%s\", \"count\": %lld, \"day\": %lld, \"days\": %lld, \"elem_bytes\": %u, "
                "\"frequency\": %.17g}\n",
                magics[k], static_cast<long long>(h.count), static_cast<long long>(h.day),
                static_cast<long long>(h.days), h.elem_bytes, h.frequency);
    return 0;
  }
  die(path + ": unknown file kind");
}

}  // namespace

int main(int argc, char **argv) {
  Options o;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&](const char *name) -> std::string {
      if (i + 1 >= argc) die(std::string(name) + " needs a value");
      return argv[++i];
    };
    if (a == "--sky") o.sky = val("--sky");
    else if (a == "--days-dir") o.days_dir = val("--days-dir");
    else if (a == "--first-day") o.first_day = std::atoi(val("--first-day").c_str());
    else if (a == "--days") o.days = std::atoi(val("--days").c_str());
    else if (a == "--frequency") o.frequency = std::atof(val("--frequency").c_str());
    else if (a == "--blockage") o.blockage = std::atoi(val("--blockage").c_str()) != 0;
    else if (a == "--fold-mirrors") o.fold = true;
    else if (a == "--nccl-reduce") o.nccl_reduce = true;
    else if (a == "--gridded") o.gridded = true;
    else if (a == "--resume") o.resume = true;
    else if (a == "--fp64") o.fp64 = true;
    else if (a == "--out-dir") o.out_dir = val("--out-dir");
    else if (a == "--sum-out") o.sum_out = val("--sum-out");
    else if (a == "--devices") o.max_devices = std::atoi(val("--devices").c_str());
    else if (a == "--convert-text") o.convert_src = val("--convert-text");
    else if (a == "--to") o.convert_dst = val("--to");
    else if (a == "--text-10m") o.text_10m = true;
    else if (a == "--info") o.info = val("--info");
    else die("unknown option " + a);
  }
  auto slash = [](std::string &p) {
    if (!p.empty() && p.back() != '/') p += '/';
  };
  slash(o.days_dir);
  slash(o.out_dir);
  slash(o.convert_src);
  slash(o.convert_dst);
  if (!o.info.empty()) return info(o.info);
  if (!o.convert_src.empty()) {
    if (o.convert_dst.empty()) die("--convert-text needs --to");
    return convert(o);
  }
  if (o.sky.empty() || o.days_dir.empty()) die("--sky and --days-dir are required");
  if (o.days < 1 || o.first_day < 1) die("--days and --first-day must be >= 1");
  if (!(o.frequency > 0)) die("--frequency must be > 0");
  if (o.gridded && o.fp64) die("--gridded is split precision; it does not take --fp64");
  if (o.resume && o.out_dir.empty()) die("--resume needs --out-dir (the day images it resumes from)");
  return stream(o);
}
