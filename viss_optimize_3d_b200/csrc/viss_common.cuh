// viss_common.cuh -- shared device helpers for the sm_100a kernels.
//
// Layout in HBM used by every kernel (built by the plan, see capi.cu):
//   pixel record  double4 (l, m, n, 0)       32 B / pixel, padded to a whole tile
//   sky           float                      4 B / pixel (zero in the padding)
//   sample record double4 (u, v, w, off)     32 B / sample
//   refs          int4 (ga, gb, ge, -1)      16 B / sample (occulter rows, -1 none)
//   occulter      double4 (qx, qy, qz, thr)  32 B / occulter
//   tile cone     double4 (cx, cy, cz, rho)  32 B / pixel tile: every pixel s of
//                 the tile has |s - c| <= rho
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace viss {

// Pixels per tile: one forward tile staged in shared memory, and one warp's
// pixel set in the adjoint (32 lanes x 4 pixels).
constexpr int kTilePix = 128;

// Phase-to-fixed-point constant: t = kMagic + u.s + off lands in [2^29, 2^30)
// for |u.s + off| < 2^28 turns, where one ulp of a double is 2^-23 turn.  The
// fraction of t is then the low 23 mantissa bits, i.e. (lo32 & 0x7fffff).
// The extra half turn centres the reduced angle in [-pi, pi); see turn_angle().
constexpr double kMagic = 805306368.0 + 0.5;  // 1.5 * 2^29 + 1/2

// Bound (turns) on |u.s + off| for the split path.
constexpr double kMaxTurns = 268435456.0;  // 2^28

// Device error word layout (written with atomicOr, read by the host):
constexpr int kErrTimeout = 1;

// ----------------------------------------------------------------- mbarrier
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One-shot try: returns true when the phase with the given parity completed.
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each try_wait already suspends
// for a hardware-chosen interval), so a lost copy ends the kernel with an
// error flag instead of a hung GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint32_t limit = (1u << 22)) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try(bar, parity)) return true;
  return false;
}

// Bulk (TMA engine) copy global -> shared, completion counted on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, uint32_t bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst_smem)),
      "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ------------------------------------------------------------- phase helpers
// Reduced angle (radians, [-pi, pi)) from t = kMagic + phase: the low 23
// mantissa bits of t are frac(phase + 1/2) in units of 2^-23 turn; placed
// under the exponent of 1.0f (one LOP3: (lo & 0x7fffff) | 0x3f800000) they
// give f in [1, 2), and 2 pi f - 3 pi is the phase reduced mod one turn.
__device__ __forceinline__ float turn_angle(double t) {
  const uint32_t lo = static_cast<uint32_t>(__double2loint(t));
  uint32_t bits;
  asm("lop3.b32 %0, %1, %2, %3, 0xEA;" : "=r"(bits) : "r"(lo), "r"(0x007fffffu), "r"(0x3f800000u));
  return fmaf(__uint_as_float(bits), 6.28318530717958648f, -9.42477796076937972f);
}

// SFU sine and cosine of an angle in [-pi, pi) (flush-to-zero variants: the
// reduced angle is never subnormal in a way that matters, and .ftz avoids the
// subnormal fix-up instructions).
__device__ __forceinline__ void sfu_sincos(float a, float &s, float &c) {
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(s) : "f"(a));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(c) : "f"(a));
}

// Exact-op-order dot product used by the occultation predicate (the oracle
// evaluates the same IEEE operations).
__device__ __forceinline__ double dot_exact(double s0, double s1, double s2, const double4 &q) {
  return __fma_rn(s2, q.z, __fma_rn(s1, q.y, __dmul_rn(s0, q.x)));
}

// Tile-vs-occulter classification.  Returns 2 if every pixel of the tile is
// visible, 0 if none is, 1 if the tile must be tested pixel by pixel.  The
// bound |s.q - c.q| <= |s - c| <= rho holds for every pixel; kConeEps covers
// the rounding of the per-pixel dot product and of c.q.
constexpr double kConeEps = 1e-12;
__device__ __forceinline__ int cone_state(const double4 &cone, const double4 &q) {
  const double d = cone.x * q.x + cone.y * q.y + cone.z * q.z;
  if (d - cone.w - kConeEps >= q.w) return 2;
  if (d + cone.w + kConeEps < q.w) return 0;
  return 1;
}

}  // namespace viss
