// formation.cu -- forward and adjoint for a satellite formation.
//
// The reference generates every baseline of a snapshot from the satellite
// positions (u = (P_a - P_b) / lambda for all pairs a < b of the S satellites)
// and evaluates each (sample, pixel) exponential separately
// (healpix_moonback_viss and computeC, vissgen3d_blockage.cu:76-102,167-192).
// The exponential factors per satellite:
//
//   e^{-2 pi i u_ab.s} = E_a(s) conj(E_b(s)),   E_a(s) = e^{-2 pi i U_a.s},
//
// with U_a = (P_a - c) / lambda for any common origin c.  So one snapshot needs
// S exponentials per pixel for its S(S-1)/2 samples, and the occultation mask
// of a pair is the product of the satellites' masks (vissgen3d_blockage.cu:88-94:
// visible iff visible from both):
//
//   forward  V_ab = e^{-2 pi i off_ab} sum_j I_j mE_j F_a(s_j) conj(F_b(s_j)),
//            F_a = m_a E_a
//   adjoint  C_j = sum_t mE_j Re( sum_{a<b} c'_ab conj(F_a(s_j)) F_b(s_j) ),
//            c'_ab = c_ab e^{+2 pi i off_ab}
//
// (mE: the snapshot's own row, the Earth cap).  The exponentials are the split
// precision path's (FP64 phase reduced to a 2^-23-turn fixed point, SFU sin /
// cos); the S(S-1)/2 complex products per pixel are FP32 FMAs.  Per 45 samples
// (S = 10) a pixel costs 10 exponentials instead of 45: the kernels are bound
// by FMA issue, not by the SFU.  The masks use the same exact FP64 predicate
// and FP32 tile classification as the direct kernels (visibility.cu).
#include "visibility.cuh"

namespace viss {

namespace {

__device__ __forceinline__ float sky_bits(const double4 &p) { return __int_as_float(__double2loint(p.w)); }

__device__ __forceinline__ bool visible_row(const double4 &q, double x, double y, double z) {
  return dot_exact(x, y, z, q) >= q.w;
}

__device__ __forceinline__ void kahan(float &s, float &c, float x) {
  const float y = __fsub_rn(x, c);
  const float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

// Index of pair (a, b), a < b, in lexicographic order.
template <int S>
__host__ __device__ constexpr int pair_index(int a, int b) {
  return a * S - a * (a + 1) / 2 + (b - a - 1);
}

// E = e^{-2 pi i U.s} as (cos, -sin) of the reduced angle.
__device__ __forceinline__ void sat_exp(const double4 &U, double x, double y, double z, float &c,
                                        float &s) {
  const double t = fma(U.z, z, fma(U.y, y, fma(U.x, x, kMagic)));
  sfu_sincos(turn_angle(t), s, c);
}

// Lane-parallel classification of one cone against the snapshot's rows (lane a
// < S: satellite a, lane S: the snapshot's row).  Returns warp-uniform masks.
template <int S>
__device__ __forceinline__ void classify(const float4 &cone, const float4 *row32, int sat_rows,
                                         int snap_rows, unsigned &hid, unsigned &mix,
                                         bool &snap_hidden) {
  const int lane = threadIdx.x & 31;
  int st = 2;
  if (lane < S && sat_rows) st = cone_state32(cone, row32[lane]);
  if (lane == S && snap_rows) st = cone_state32(cone, row32[S]);
  hid = __ballot_sync(0xffffffffu, lane < S && st == 0);
  mix = __ballot_sync(0xffffffffu, lane <= S && st == 1);
  snap_hidden = __ballot_sync(0xffffffffu, lane == S && st == 0) != 0;
}

}  // namespace

// --------------------------------------------------------------- forward
// A warp owns one snapshot and accumulates its S(S-1)/2 samples over a chunk
// of pixel tiles (lane = pixel within each 32-pixel group); the CTA's warps
// share the staged tiles (the stage ring of the direct forward).  Per-lane
// FP32 sums cover at most kFormFoldTiles * 4 = 128 pixels; they are then
// summed over the warp and added to FP64 accumulators (lane l keeps pairs l,
// l + 32, l + 64).
//
// Tile modes (warp-uniform, from the classification): kOpen -- every row sees
// the whole tile, no mask arithmetic; kMixed -- the general case: satellites
// that see none of it are zeroed by a uniform factor, rows that see part of
// it take the exact per-pixel predicate.
enum FormMode { kOpen = 0, kMixed = 1 };

template <int S, int MODE>
__device__ __forceinline__ void form_fwd_tile(const double4 *tp, const double4 *U,
                                              const double4 *rows, unsigned hid, unsigned mix,
                                              float (&ar)[form_pairs(S)],
                                              float (&ai)[form_pairs(S)]) {
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int q = 0; q < kTilePix / 32; ++q) {
    const double4 rec = tp[q * 32 + lane];
    const double x = rec.x, y = rec.y, z = rec.z;
    float I = sky_bits(rec);
    if (MODE == kMixed && ((mix >> S) & 1u)) I = visible_row(rows[S], x, y, z) ? I : 0.f;
    float Gr[S - 1], Gi[S - 1];
#pragma unroll
    for (int b = 0; b < S; ++b) {
      float c, s;
      sat_exp(U[b], x, y, z, c, s);
      float Fr = c, Fi = -s;                 // F_b = m e^{-i theta}
      if (MODE != kOpen) {
        float m = ((hid >> b) & 1u) ? 0.f : 1.f;
        if (MODE == kMixed && ((mix >> b) & 1u)) m = visible_row(rows[b], x, y, z) ? m : 0.f;
        Fr *= m;
        Fi *= m;
      }
      const float cr = Fr, ci = -Fi;         // conj(F_b)
#pragma unroll
      for (int a = 0; a < b; ++a) {
        const int pi = pair_index<S>(a, b);
        ar[pi] = fmaf(Gr[a], cr, fmaf(-Gi[a], ci, ar[pi]));
        ai[pi] = fmaf(Gr[a], ci, fmaf(Gi[a], cr, ai[pi]));
      }
      if (b < S - 1) {
        Gr[b] = I * Fr;
        Gi[b] = I * Fi;
      }
    }
  }
}

template <int S>
__global__ void __launch_bounds__(kFormFwdNT, 1) k_form_forward(const FormParams p) {
  constexpr int B = form_pairs(S);
  constexpr int NW = kFormFwdNT / 32;
  constexpr int ST = kFwdStages;
  __shared__ __align__(128) double4 s_pix[ST][kTilePix];
  __shared__ __align__(16) double4 s_U[NW][S];
  __shared__ __align__(16) double4 s_row[NW][S + 1];
  __shared__ __align__(16) float4 s_row32[NW][S + 1];
  __shared__ __align__(8) uint64_t s_full[ST], s_empty[ST];
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // a CTA never straddles channels: blockIdx.x = channel * blocks_per_channel + block
  const long long bpc = (p.Tc + NW - 1) / NW;
  const long long ch = blockIdx.x / bpc;
  const long long tl = (blockIdx.x - ch * bpc) * NW + warp;
  const bool tok = tl < p.Tc;
  const long long t = ch * p.Tc + tl;
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  if (lane < S) s_U[warp][lane] = tok ? p.U[t * S + lane] : make_double4(0, 0, 0, 0);
  if (lane <= S) {
    double4 r = pass;
    if (tok && lane < S && p.sat_rows) r = p.occ[t * S + lane];
    if (tok && lane == S && p.snap_rows) r = p.occ[p.T * S + t];
    s_row[warp][lane] = r;
    float4 r32 = make_float4(0.f, 0.f, 0.f, -4.f);
    if (tok && lane < S && p.sat_rows) r32 = p.occ32[t * S + lane];
    if (tok && lane == S && p.snap_rows) r32 = p.occ32[p.T * S + t];
    s_row32[warp][lane] = r32;
  }

  const int t0 = blockIdx.y * p.tiles_per_chunk;
  const int ntile = max(0, min(t0 + p.tiles_per_chunk, p.ntiles) - t0);
  constexpr uint32_t kTileBytes = kTilePix * sizeof(double4);
  const double4 *pix = p.pix + ch * p.Jpad;  // this channel's sky records
  auto issue = [&](int i, int stage) {
    mbar_expect_tx(&s_full[stage], kTileBytes);
    bulk_g2s(s_pix[stage], pix + static_cast<long long>(t0 + i) * kTilePix, kTileBytes,
             &s_full[stage]);
  };
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < ST; ++s) {
      mbar_init(&s_full[s], 1);
      mbar_init(&s_empty[s], NW);
    }
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  float ar[B], ai[B];
#pragma unroll
  for (int k = 0; k < B; ++k) ar[k] = ai[k] = 0.f;
  double sr[(B + 31) / 32], si[(B + 31) / 32];
#pragma unroll
  for (int k = 0; k < (B + 31) / 32; ++k) sr[k] = si[k] = 0.0;
  auto fold = [&]() {
#pragma unroll
    for (int k = 0; k < B; ++k) {
      float vr = ar[k], vi = ai[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        vr += __shfl_xor_sync(0xffffffffu, vr, o);
        vi += __shfl_xor_sync(0xffffffffu, vi, o);
      }
      if (lane == (k & 31)) {
        sr[k >> 5] += vr;
        si[k >> 5] += vi;
      }
      ar[k] = ai[k] = 0.f;
    }
  };

  unsigned long long evaluated = 0, mixed_terms = 0;
  int next = 0, since_fold = 0;
  for (int it = 0; it < ntile; ++it) {
    const int tt = t0 + it, stage = it % ST;
    if (tid == 0 && !ring_refill<ST>(s_empty, next, it, ntile, issue)) {
      atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
    }
    if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
    unsigned hid, mix;
    bool snap_hidden;
    classify<S>(p.cones[tt], s_row32[warp], p.sat_rows, p.snap_rows, hid, mix, snap_hidden);
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_full[stage], static_cast<uint32_t>(it / ST) & 1u))) {
      if (lane == 0) atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
      break;
    }
    // a pair needs both satellites: skip the tile unless two see some of it
    if (tok && !snap_hidden && S - __popc(hid) >= 2) {
      if (mix | hid) {
        form_fwd_tile<S, kMixed>(s_pix[stage], s_U[warp], s_row[warp], hid, mix, ar, ai);
        mixed_terms += static_cast<unsigned long long>(kTilePix) * B;
      } else {
        form_fwd_tile<S, kOpen>(s_pix[stage], s_U[warp], s_row[warp], hid, mix, ar, ai);
      }
      evaluated += static_cast<unsigned long long>(kTilePix) * B;
    }
    ring_release(s_empty, stage);
    if (++since_fold == kFormFoldTiles) {
      fold();
      since_fold = 0;
    }
  }
  if (tid == 0) ring_drain<ST>(s_full, next);
  fold();
  if (p.counter && lane == 0) {
    if (evaluated) atomicAdd(p.counter, evaluated);
    if (mixed_terms) atomicAdd(p.counter + 2, mixed_terms);
  }
  if (!tok) return;
  double2 *out = p.part_fwd + static_cast<long long>(blockIdx.y) * p.T * B + t * B;
#pragma unroll
  for (int k = 0; k < (B + 31) / 32; ++k) {
    const int pi = lane + 32 * k;
    if (pi < B) out[pi] = make_double2(sr[k], si[k]);
  }
}

// --------------------------------------------------------------- adjoint
// A warp owns 32 * P pixels (P per lane); the CTA streams a chunk of
// snapshots through a shared-memory ring, kFormSnapTile snapshots per stage
// (satellite vectors, coefficients and occulter rows, by bulk copies).  Per
// pixel and snapshot: Q = sum_b Re(H_b F_b), H_b = sum_{a<b} c'_ab conj(F_a).
// FP32 sums over one staged tile, Kahan-folded per tile, FP64 across chunks.
constexpr int kFormAdjP = 2;

template <int S>
struct FormAdjStage {
  double4 U[kFormSnapTile * S];
  double4 rows[kFormSnapTile * S];
  double4 snap[kFormSnapTile];
  float4 rows32[kFormSnapTile * S];
  float4 snap32[kFormSnapTile];
  float2 coef[kFormSnapTile * form_coef_stride(S)];
};

// Q[q] (one snapshot) for the lane's P pixels; cf is the snapshot's column
// layout of coefficients (form_col0), U its satellite vectors.
template <int S, int P, int MODE>
__device__ __forceinline__ void form_adj_snapshot(const double4 *U, const float2 *cf,
                                                  const double4 *rows, unsigned hid, unsigned mix,
                                                  const double (&sx)[P], const double (&sy)[P],
                                                  const double (&sz)[P], float (&Q)[P]) {
  float Kr[S - 1][P], Ki[S - 1][P];
#pragma unroll
  for (int q = 0; q < P; ++q) Q[q] = 0.f;
#pragma unroll
  for (int b = 0; b < S; ++b) {
    const double4 Ub = U[b];
    float Fr[P], Fi[P];
#pragma unroll
    for (int q = 0; q < P; ++q) {
      float c, s;
      sat_exp(Ub, sx[q], sy[q], sz[q], c, s);
      Fr[q] = c;
      Fi[q] = -s;
      if (MODE != kOpen) {
        float m = ((hid >> b) & 1u) ? 0.f : 1.f;
        if (MODE == kMixed && ((mix >> b) & 1u)) m = visible_row(rows[b], sx[q], sy[q], sz[q]) ? m : 0.f;
        Fr[q] *= m;
        Fi[q] *= m;
      }
    }
    if (b > 0) {
      float Hr[P], Hi[P];
#pragma unroll
      for (int q = 0; q < P; ++q) Hr[q] = Hi[q] = 0.f;
      const float4 *col = reinterpret_cast<const float4 *>(cf + form_col0(b));
#pragma unroll
      for (int a2 = 0; a2 < b; a2 += 2) {
        const float4 c2 = col[a2 / 2];  // coefficients of pairs (a2, b) and (a2 + 1, b)
#pragma unroll
        for (int q = 0; q < P; ++q) {
          Hr[q] = fmaf(c2.x, Kr[a2][q], fmaf(-c2.y, Ki[a2][q], Hr[q]));
          Hi[q] = fmaf(c2.x, Ki[a2][q], fmaf(c2.y, Kr[a2][q], Hi[q]));
        }
        if (a2 + 1 < b) {
#pragma unroll
          for (int q = 0; q < P; ++q) {
            Hr[q] = fmaf(c2.z, Kr[a2 + 1][q], fmaf(-c2.w, Ki[a2 + 1][q], Hr[q]));
            Hi[q] = fmaf(c2.z, Ki[a2 + 1][q], fmaf(c2.w, Kr[a2 + 1][q], Hi[q]));
          }
        }
      }
#pragma unroll
      for (int q = 0; q < P; ++q) Q[q] = fmaf(Hr[q], Fr[q], fmaf(-Hi[q], Fi[q], Q[q]));
    }
    if (b < S - 1) {
#pragma unroll
      for (int q = 0; q < P; ++q) {
        Kr[b][q] = Fr[q];
        Ki[b][q] = -Fi[q];
      }
    }
  }
}

template <int S>
__global__ void __launch_bounds__(kFormAdjNT, 1) k_form_adjoint(const FormParams p) {
  constexpr int CB = form_coef_stride(S);
  constexpr int NW = kFormAdjNT / 32;
  constexpr int ST = 3;
  constexpr int P = kFormAdjP;
  __shared__ __align__(128) FormAdjStage<S> s_stage[ST];
  __shared__ __align__(8) uint64_t s_full[ST], s_empty[ST];
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long wpix = (static_cast<long long>(blockIdx.x) * NW + warp) * (32 * P);
  const bool tile_ok = wpix < p.Jpad;
  double sx[P], sy[P], sz[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const double4 v = tile_ok ? p.pix[wpix + 32 * q + lane] : make_double4(0, 0, 1, 0);
    sx[q] = v.x; sy[q] = v.y; sz[q] = v.z;
  }
  // the warp's pixels lie in one kTilePix tile (32 P divides kTilePix)
  const float4 cone = tile_ok ? p.cones[wpix / kTilePix] : make_float4(0.f, 0.f, 1.f, 4.f);

  // blockIdx.y = channel * nchunk + chunk; a chunk never leaves its channel
  const long long ch = blockIdx.y / p.nchunk;
  const long long s0 = ch * p.Tc + static_cast<long long>(blockIdx.y - ch * p.nchunk) * p.snaps_per_chunk;
  const long long s1 = min(s0 + p.snaps_per_chunk, (ch + 1) * p.Tc);
  const int ntile = static_cast<int>((max(0LL, s1 - s0) + kFormSnapTile - 1) / kFormSnapTile);
  auto issue = [&](int i, int stage) {
    const long long ts = s0 + static_cast<long long>(i) * kFormSnapTile;
    const int n = static_cast<int>(min(static_cast<long long>(kFormSnapTile), s1 - ts));
    FormAdjStage<S> &g = s_stage[stage];
    uint32_t bytes = n * S * 32u + n * CB * 8u;
    if (p.sat_rows) bytes += n * S * (32u + 16u);
    if (p.snap_rows) bytes += n * (32u + 16u);
    mbar_expect_tx(&s_full[stage], bytes);
    bulk_g2s(g.U, p.U + ts * S, n * S * 32u, &s_full[stage]);
    bulk_g2s(g.coef, p.coef + ts * CB, n * CB * 8u, &s_full[stage]);
    if (p.sat_rows) {
      bulk_g2s(g.rows, p.occ + ts * S, n * S * 32u, &s_full[stage]);
      bulk_g2s(g.rows32, p.occ32 + ts * S, n * S * 16u, &s_full[stage]);
    }
    if (p.snap_rows) {
      bulk_g2s(g.snap, p.occ + p.T * S + ts, n * 32u, &s_full[stage]);
      bulk_g2s(g.snap32, p.occ32 + p.T * S + ts, n * 16u, &s_full[stage]);
    }
  };
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < ST; ++s) {
      mbar_init(&s_full[s], 1);
      mbar_init(&s_empty[s], NW);
    }
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  float ks[P], kc[P];
#pragma unroll
  for (int q = 0; q < P; ++q) ks[q] = kc[q] = 0.f;
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  unsigned long long evaluated = 0, mixed_terms = 0;
  int next = 0;
  for (int it = 0; it < ntile; ++it) {
    const int stage = it % ST;
    if (tid == 0 && !ring_refill<ST>(s_empty, next, it, ntile, issue)) {
      atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
    }
    if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_full[stage], static_cast<uint32_t>(it / ST) & 1u))) {
      if (lane == 0) atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
      break;
    }
    const FormAdjStage<S> &g = s_stage[stage];
    const long long ts = s0 + static_cast<long long>(it) * kFormSnapTile;
    const int n = static_cast<int>(min(static_cast<long long>(kFormSnapTile), s1 - ts));
    float acc[P];
#pragma unroll
    for (int q = 0; q < P; ++q) acc[q] = 0.f;
#pragma unroll 1
    for (int k = 0; k < n; ++k) {
      // classify the warp's tile against this snapshot's rows (lane-parallel)
      int st = 2;
      if (lane < S && p.sat_rows) st = cone_state32(cone, g.rows32[k * S + lane]);
      if (lane == S && p.snap_rows) st = cone_state32(cone, g.snap32[k]);
      const unsigned hid = __ballot_sync(0xffffffffu, lane < S && st == 0);
      const unsigned mix = __ballot_sync(0xffffffffu, lane <= S && st == 1);
      const bool snap_hidden = __ballot_sync(0xffffffffu, lane == S && st == 0) != 0;
      if (!tile_ok || snap_hidden || S - __popc(hid) < 2) continue;
      evaluated += static_cast<unsigned long long>(32 * P) * form_pairs(S);
      float Q[P];
      // two code paths only: a third (hidden satellites without mixed rows)
      // measured slower, the unrolled bodies competing for instruction cache
      if (mix | hid) {
        mixed_terms += static_cast<unsigned long long>(32 * P) * form_pairs(S);
        form_adj_snapshot<S, P, kMixed>(g.U + k * S, g.coef + k * CB, g.rows + k * S, hid, mix, sx, sy, sz, Q);
        if ((mix >> S) & 1u) {
          const double4 re = p.snap_rows ? g.snap[k] : pass;
#pragma unroll
          for (int q = 0; q < P; ++q)
            if (!visible_row(re, sx[q], sy[q], sz[q])) Q[q] = 0.f;
        }
      } else {
        form_adj_snapshot<S, P, kOpen>(g.U + k * S, g.coef + k * CB, g.rows + k * S, hid, mix, sx, sy, sz, Q);
      }
#pragma unroll
      for (int q = 0; q < P; ++q) acc[q] += Q[q];
    }
#pragma unroll
    for (int q = 0; q < P; ++q) kahan(ks[q], kc[q], acc[q]);
    ring_release(s_empty, stage);
  }
  if (tid == 0) ring_drain<ST>(s_full, next);
  if (p.counter && lane == 0) {
    if (evaluated) atomicAdd(p.counter, evaluated);
    if (mixed_terms) atomicAdd(p.counter + 2, mixed_terms);
  }
  if (!tile_ok) return;
  double *out = p.part_adj + static_cast<long long>(blockIdx.y) * p.Jpad;
#pragma unroll
  for (int q = 0; q < P; ++q)
    out[wpix + 32 * q + lane] = static_cast<double>(ks[q]) - static_cast<double>(kc[q]);
}

int form_adjoint_pixels_per_block() { return (kFormAdjNT / 32) * 32 * kFormAdjP; }

template <int S>
static cudaError_t form_fwd_inst(const FormParams &p, int nchunk, cudaStream_t st) {
  const long long gx = p.channels * ((p.Tc + kFormFwdNT / 32 - 1) / (kFormFwdNT / 32));
  if (gx > 0x7fffffffLL || nchunk > 65535) return cudaErrorInvalidValue;
  k_form_forward<S><<<dim3(static_cast<unsigned>(gx), nchunk), kFormFwdNT, 0, st>>>(p);
  return cudaGetLastError();
}

template <int S>
static cudaError_t form_adj_inst(const FormParams &p, int nchunk, cudaStream_t st) {
  const long long gx = (p.Jpad + form_adjoint_pixels_per_block() - 1) / form_adjoint_pixels_per_block();
  const long long gy = static_cast<long long>(p.channels) * nchunk;
  if (gy > 65535) return cudaErrorInvalidValue;
  k_form_adjoint<S><<<dim3(static_cast<unsigned>(gx), static_cast<unsigned>(gy)), kFormAdjNT, 0, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_form_forward(const FormParams &p, int S, int nchunk, cudaStream_t st) {
  if (p.T <= 0 || p.ntiles <= 0) return cudaSuccess;
  if (p.channels < 1 || p.Tc * p.channels != p.T) return cudaErrorInvalidValue;
  switch (S) {
    case 2: return form_fwd_inst<2>(p, nchunk, st);
    case 3: return form_fwd_inst<3>(p, nchunk, st);
    case 4: return form_fwd_inst<4>(p, nchunk, st);
    case 5: return form_fwd_inst<5>(p, nchunk, st);
    case 6: return form_fwd_inst<6>(p, nchunk, st);
    case 7: return form_fwd_inst<7>(p, nchunk, st);
    case 8: return form_fwd_inst<8>(p, nchunk, st);
    case 9: return form_fwd_inst<9>(p, nchunk, st);
    case 10: return form_fwd_inst<10>(p, nchunk, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_form_adjoint(const FormParams &p, int S, int nchunk, cudaStream_t st) {
  if (p.T <= 0 || p.Jpad <= 0) return cudaSuccess;
  if (p.channels < 1 || p.Tc * p.channels != p.T) return cudaErrorInvalidValue;
  switch (S) {
    case 2: return form_adj_inst<2>(p, nchunk, st);
    case 3: return form_adj_inst<3>(p, nchunk, st);
    case 4: return form_adj_inst<4>(p, nchunk, st);
    case 5: return form_adj_inst<5>(p, nchunk, st);
    case 6: return form_adj_inst<6>(p, nchunk, st);
    case 7: return form_adj_inst<7>(p, nchunk, st);
    case 8: return form_adj_inst<8>(p, nchunk, st);
    case 9: return form_adj_inst<9>(p, nchunk, st);
    case 10: return form_adj_inst<10>(p, nchunk, st);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ staging
// U rows (T*S x 3 FP64) -> double4; the bound |Ux| + |Uy| + |Uz| + |off| over
// everything (>= |U_a.s + off| for unit s), non-finite -> +inf.
__global__ void k_form_stage_U(long long n, const double *U, double4 *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(U[3 * i], U[3 * i + 1], U[3 * i + 2], 0.0);
}

__global__ void k_form_bound(long long n, const double *U, long long m, const double *off,
                             unsigned long long *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  double b = 0;
  if (i < n) b = fabs(U[3 * i]) + fabs(U[3 * i + 1]) + fabs(U[3 * i + 2]);
  if (off && i < m) b = fmax(b, fabs(off[i]));
  if (!(b <= 1e300)) b = __longlong_as_double(0x7ff0000000000000ll);
  for (int o = 16; o > 0; o >>= 1) b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, static_cast<unsigned long long>(__double_as_longlong(b)));
}

// c'[t][form_col0(b) + a] = c[t B + pair(a, b)] e^{+2 pi i off} (FP64
// rotation), zero in the padding of each column.
__global__ void k_form_stage_coef(long long T, int S, int CB, const float2 *coef, const double *off,
                                  float2 *out) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= T * CB) return;
  const long long t = i / CB;
  const int r = static_cast<int>(i - t * CB);
  int b = 1;
  while (b + 1 < S && form_col0(b + 1) <= r) ++b;
  const int a = r - form_col0(b);
  if (a >= b) {
    out[i] = make_float2(0.f, 0.f);
    return;
  }
  const long long k = t * form_pairs(S) + (a * S - a * (a + 1) / 2 + (b - a - 1));
  const float2 c = coef[k];
  if (!off) {
    out[i] = c;
    return;
  }
  const double o = off[k];
  double sn, cs;
  sincospi(2.0 * (o - rint(o)), &sn, &cs);
  const double re = c.x, im = c.y;
  out[i] = make_float2(static_cast<float>(re * cs - im * sn), static_cast<float>(re * sn + im * cs));
}

// V_k = e^{-2 pi i off_k} sum over chunks (FP64), optionally accumulated.
__global__ void k_form_reduce_fwd(long long K, int nchunk, const double2 *part, const double *off,
                                  float2 *V, int accumulate) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double re = 0, im = 0;
  for (int c = 0; c < nchunk; ++c) {
    const double2 v = part[static_cast<long long>(c) * K + k];
    re += v.x;
    im += v.y;
  }
  if (off) {
    const double o = off[k];
    double sn, cs;
    sincospi(2.0 * (o - rint(o)), &sn, &cs);
    const double r = re * cs + im * sn, i = im * cs - re * sn;
    re = r;
    im = i;
  }
  if (accumulate) {
    const float2 v = V[k];
    re += v.x;
    im += v.y;
  }
  V[k] = make_float2(static_cast<float>(re), static_cast<float>(im));
}

static inline unsigned nblk(long long n, int bs) { return static_cast<unsigned>((n + bs - 1) / bs); }

cudaError_t launch_form_stage(long long T, int S, const double *U, const double *off,
                              double4 *U4, unsigned long long *bound, cudaStream_t st) {
  const long long n = T * S, m = off ? T * form_pairs(S) : 0;
  k_form_stage_U<<<nblk(n, 256), 256, 0, st>>>(n, U, U4);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_form_bound<<<nblk(n > m ? n : m, 256), 256, 0, st>>>(n, U, m, off, bound);
  return cudaGetLastError();
}

cudaError_t launch_form_stage_coef(long long T, int S, const float2 *coef, const double *off,
                                   float2 *out, cudaStream_t st) {
  const int CB = form_coef_stride(S);
  k_form_stage_coef<<<nblk(T * CB, 256), 256, 0, st>>>(T, S, CB, coef, off, out);
  return cudaGetLastError();
}

cudaError_t launch_form_reduce_fwd(long long K, int nchunk, const double2 *part, const double *off,
                                   float2 *V, int acc, cudaStream_t st) {
  if (K <= 0) return cudaSuccess;
  k_form_reduce_fwd<<<nblk(K, 256), 256, 0, st>>>(K, nchunk, part, off, V, acc);
  return cudaGetLastError();
}

}  // namespace viss
