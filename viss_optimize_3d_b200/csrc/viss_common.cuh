// viss_common.cuh -- shared device helpers for the sm_100a kernels.
//
// Layout in HBM used by every kernel (built by the plan, see capi.cu):
//   pixel record  double4 (l, m, n, 0)       32 B / pixel, padded to a whole tile
//   sky           float                      4 B / pixel (zero in the padding)
//   sample record double4 (u, v, w, off)     32 B / sample
//   refs          int4 (ga, gb, ge, -1)      16 B / sample (occulter rows, -1 none)
//   occulter      double4 (qx, qy, qz, thr)  32 B / occulter (exact test)
//   occulter32    float4 (q, thr) / |q|      16 B / occulter (classification)
//   cones         float4 (cx, cy, cz, w)     16 B per pixel tile, then 4 x 16 B
//                 per tile for its 32-pixel sub-tiles, then 16 B per super-tile of
//                 kSuperTiles tiles (see cone_state32 and cone_count)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace viss {

// Pixels per tile: one forward tile staged in shared memory, and one warp's
// pixel set in the adjoint (32 lanes x 4 pixels).
constexpr int kTilePix = 128;

// Tiles per super-tile: the forward classifies a sample once per super-tile
// and skips the per-tile test where the super-tile is wholly visible or
// wholly hidden for it.
constexpr int kSuperTiles = 8;

// float4 entries of the cone array for ntiles tiles: tile cones [0, nt),
// sub-tile cones [nt, 5 nt), super-tile cones [5 nt, 5 nt + ceil(nt / 8)).
__host__ __device__ constexpr long long cone_count(long long ntiles) {
  return 5 * ntiles + (ntiles + kSuperTiles - 1) / kSuperTiles;
}

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

// Arrive (count one) on a barrier without waiting.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// One-shot try: returns true when the phase with the given parity completed
// (may suspend the thread for a hardware-chosen interval first).
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

// Non-blocking test of the same condition.
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait: gives up after `limit_ns` nanoseconds of the global timer (or
// 2^26 polls, whichever comes first), so a lost copy or a stalled peer warp
// ends the kernel with an error flag instead of a hung GPU.  The default
// limit is far above any legitimate wait in these kernels (one tile of work).
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // 1 s
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t start = global_ns();
  for (uint32_t i = 0; i < (1u << 20); ++i) {
#pragma unroll 1
    for (int j = 0; j < 64; ++j)
      if (mbar_try(bar, parity)) return true;
    if (global_ns() - start > limit_ns) return false;
  }
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

// --------------------------------------------------------------- stage ring
// An S-stage ring of shared-memory tiles filled by bulk copies.  full[s]
// (count 1) completes when the tile in stage s has landed; empty[s] (count =
// the CTA's warps) completes when every warp has released it.  Tile i lives
// in stage i % S and is phase (i / S) & 1 of both barriers.  One thread (the
// producer, itself a consumer in warp 0) refills stages as they free up, so
// warps drift up to S - 1 tiles apart instead of meeting at a CTA barrier
// after every tile.

// Producer: issue tiles [next, min(ntile, it + S)) in order through
// issue(i, stage).  A stage still held by a slower warp stops the refill
// (retried at the producer's next tile) unless it is needed for tile `it`,
// the one the producer's own warp consumes now, which is waited for
// (bounded).  Returns false on a timeout.
template <int S, typename Issue>
__device__ __forceinline__ bool ring_refill(uint64_t *empty, int &next, int it, int ntile,
                                            Issue &&issue) {
  while (next < ntile && next < it + S) {
    const int s = next % S;
    if (next >= S) {
      const uint32_t par = static_cast<uint32_t>(next / S - 1) & 1u;
      if (next == it) {
        if (!mbar_wait_bounded(&empty[s], par)) return false;
      } else if (!mbar_test(&empty[s], par)) {
        break;
      }
    }
    issue(next, s);
    ++next;
  }
  return true;
}

// Consumer: the calling warp is done reading stage s.
__device__ __forceinline__ void ring_release(uint64_t *empty, int s) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive(&empty[s]);
}

// Producer, before the CTA exits: let every copy still in flight land, bounded.
// Tile i is issued only after tile i - S was consumed, so only the last S
// issued tiles can still be in flight.
template <int S>
__device__ __forceinline__ void ring_drain(uint64_t *full, int next) {
  for (int i = next > S ? next - S : 0; i < next; ++i)
    mbar_wait_bounded(&full[i % S], static_cast<uint32_t>(i / S) & 1u);
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

// Tile-vs-occulter classification, in FP32 (it only has to be conservative:
// the exact FP64 predicate decides every pixel it leaves open).
//   cone  float4 (cx, cy, cz, w): unit centre c rounded to FP32, and w >= the
//         largest |s - c| over the tile's pixels s, plus kConeMargin32
//   row   float4 (qx, qy, qz, thr) / |q|: the occulter row scaled to a unit
//         direction (the same half-space), rounded to FP32
// Returns 2 if every pixel of the tile is visible, 0 if none is, 1 if the tile
// must be tested pixel by pixel.  For a unit q, |s.q - c.q| <= |s - c|;
// kConeMargin32 covers the FP32 roundings (dot product ~2e-7, row and
// threshold rounding ~2e-7, the +-w below ~2e-7) with a wide safety factor.
// NaN rows or cones compare false both ways: "test every pixel".
constexpr double kConeMargin32 = 4e-6;
__device__ __forceinline__ int cone_state32(const float4 &cone, const float4 &q) {
  const float d = fmaf(cone.z, q.z, fmaf(cone.y, q.y, cone.x * q.x));
  if (d - cone.w >= q.w) return 2;
  if (d + cone.w < q.w) return 0;
  return 1;
}

// A sample (occulter refs rf, -1 = none) sees every pixel of a cone: each of
// its rows classifies the cone as wholly visible.  The gridded adjoint's
// spreading and the direct adjoint's hybrid instance both decide with this
// one function on the same stored cone and rows, so each (sample, facet) pair
// is taken by exactly one of them.
__device__ __forceinline__ bool facet_open(const int4 &rf, const float4 &cone, const float4 *occ32) {
  return (rf.x < 0 || cone_state32(cone, occ32[rf.x]) == 2) && (rf.y < 0 || cone_state32(cone, occ32[rf.y]) == 2) &&
         (rf.z < 0 || cone_state32(cone, occ32[rf.z]) == 2);
}

}  // namespace viss
