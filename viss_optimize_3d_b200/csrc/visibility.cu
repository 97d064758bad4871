// visibility.cu -- the two O(K x J) kernels of the hot path.
//
//   forward  V_k = sum_j I_j vis_kj exp(-2 pi i (u_k.s_j + off_k))
//            replaces healpix_moonback_viss (vissgen3d_blockage.cu:76-102)
//   adjoint  C_j = sum_k Re(a_k exp(+2 pi i (u_k.s_j + off_k))) vis_kj
//            replaces computeC (vissgen3d_blockage.cu:167-192)
//
// Both are matrix-free matvecs bound by the SFU (two MUFU ops per term: sin
// and cos), not by HBM and not by tensor cores.  Per term the split path
// issues 3 DFMA (phase in FP64, already reduced to a 2^-23-turn fixed point by
// the kMagic offset), 1 LOP3 (fraction -> float), 1 FFMA (-> radians), the
// SFU's argument scaling, sin, cos and 2 FFMA (accumulate).
//
// Work decomposition
//   forward: a CTA owns NT*R samples (R per thread, in registers) and one
//            chunk of pixel tiles; tiles of kTilePix pixel records stream
//            through a 2-deep shared-memory ring filled by cp.async.bulk
//            (TMA engine) and are read as warp-wide broadcasts.  Partial sums
//            of each chunk go to a [chunk][K] FP64 workspace; k_reduce_fwd
//            adds the chunks in FP64.
//   adjoint: a warp owns 32*P pixels (P per lane, in registers); a CTA owns
//            NT/32 such warp tiles and one chunk of samples, which stream
//            through shared memory the same way.  Chunks go to a [chunk][Jpad]
//            FP64 workspace reduced (and un-permuted) by k_reduce_adj.
// Occultation: every kTilePix-pixel tile carries a bounding cone (centre,
// chord radius).  Against each of a sample's occulters a tile is "all
// visible" (no per-term test), "none visible" (the sample skips the tile) or
// "mixed" (the exact FP64 predicate per term, the same operations as the CPU
// oracle, so the mask bits match it exactly).  The decision is warp-uniform:
// the warp votes in the forward; in the adjoint the sample is uniform across
// the warp.
//
// Accuracy: terms are summed in FP32 within a tile / sample group (<= 128
// terms per accumulator), those partial sums are folded into a
// Kahan-compensated FP32 sum, and chunks are added in FP64.  The SFU's sin and
// cos carry a small mean error over a turn (~1e-8 on the B200); summed over
// all pixels it would grow with the total flux rather than with |V|, which for
// long baselines is ~700x smaller.  The split path therefore evaluates odd
// pixel records half a turn further on and negates them (e^{i(x+pi)} = -e^{ix}),
// so a constant SFU error cancels between neighbouring pixels.
#include "visibility.cuh"

namespace viss {

// Kahan-compensated add of x into (s, c).
__device__ __forceinline__ void kahan_add(float &s, float &c, float x) {
  const float y = __fsub_rn(x, c);
  const float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

// Classification of a sample (3 occulter refs) against one tile cone, packed:
// bits 0-1 state (2 every pixel visible, 0 none, 1 mixed), bits 2-4 which
// refs are mixed on this tile (only those need the per-pixel test).
__device__ __forceinline__ int sample_state(const int4 &rf, const double4 &cone,
                                            const double4 *occ) {
  int st = 2, need = 0;
  const int r3[3] = {rf.x, rf.y, rf.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (r3[c] < 0) continue;
    const int s = cone_state(cone, occ[r3[c]]);
    st = min(st, s);
    if (s == 1) need |= 1 << c;
  }
  return st == 1 ? (1 | (need << 2)) : st;
}

// The same against the union of two tiles (a warp tile of 256 pixels): hidden
// only if hidden on both; all visible only if all visible on both; otherwise
// every ref that is not all-visible on both tiles is tested per pixel.
__device__ __forceinline__ int sample_state2(const int4 &rf, const double4 &c0,
                                             const double4 &c1, const double4 *occ) {
  const int a = sample_state(rf, c0, occ), b = sample_state(rf, c1, occ);
  const int sa = a & 3, sb = b & 3;
  if (sa == 0 && sb == 0) return 0;
  if (sa == 2 && sb == 2) return 2;
  int need = 0;
  const int r3[3] = {rf.x, rf.y, rf.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (r3[c] < 0) continue;
    const bool full0 = (sa == 2) || (sa == 1 && !((a >> (2 + c)) & 1));
    const bool full1 = (sb == 2) || (sb == 1 && !((b >> (2 + c)) & 1));
    if (!(full0 && full1)) need |= 1 << c;
  }
  return need ? (1 | (need << 2)) : 2;
}

// The occulter rows a mixed sample must test; rows it need not test become a
// row every direction passes (thr = -4 < any dot of unit vectors).
__device__ __forceinline__ void mixed_rows(const int4 &rf, int code, const double4 *occ,
                                           double4 &q0, double4 &q1, double4 &q2) {
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  q0 = (code & 4) ? occ[rf.x] : pass;
  q1 = (code & 8) ? occ[rf.y] : pass;
  q2 = (code & 16) ? occ[rf.z] : pass;
}

__device__ __forceinline__ bool visible_rows(const double4 &q0, const double4 &q1,
                                             const double4 &q2, double s0, double s1, double s2) {
  return (dot_exact(s0, s1, s2, q0) >= q0.w) & (dot_exact(s0, s1, s2, q1) >= q1.w) &
         (dot_exact(s0, s1, s2, q2) >= q2.w);
}

__device__ __forceinline__ float sky_of(const double4 &p) {
  return __int_as_float(__double2loint(p.w));
}

// FP64 reference term: (sin, cos) of 2 pi (phase mod 1), phase in FP64.
__device__ __forceinline__ void sincos_turns_fp64(double t, double &sn, double &cs) {
  const double f = t - rint(t);
  sincospi(2.0 * f, &sn, &cs);
}

// One forward term into (re, im): sky I at phase t.
template <bool FP64>
__device__ __forceinline__ void fwd_term(double t, float I, float &re, float &im, double &dre,
                                         double &dim) {
  if (FP64) {
    double sn, cs;
    sincos_turns_fp64(t, sn, cs);
    dre = fma(static_cast<double>(I), cs, dre);
    dim = fma(-static_cast<double>(I), sn, dim);
  } else {
    float sn, cs;
    sfu_sincos(turn_angle(t), sn, cs);
    re = fmaf(I, cs, re);
    im = fmaf(-I, sn, im);
  }
}

// ======================================================================
// forward
// ======================================================================
template <int NT, int R, int MINB, bool MASKED, bool FP64>
__global__ void __launch_bounds__(NT, MINB) k_forward(const FwdParams p) {
  __shared__ __align__(128) double4 s_pix[2][kTilePix];
  __shared__ __align__(16) int4 s_refs[MASKED ? R : 1][MASKED ? NT : 1];
  // Kahan (sum, comp) of re and im per sample, kept in shared memory (touched
  // once per tile) so the registers hold only what the inner loop needs
  __shared__ float s_kahan[FP64 ? 1 : 4][FP64 ? 1 : R][FP64 ? 1 : NT];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  // CTAs never straddle channels: blockIdx.x = channel * blocks_per_channel + block
  const long long bpc = (p.Kc + NT * R - 1) / (NT * R);
  const long long ch = blockIdx.x / bpc;
  const long long kloc = (blockIdx.x - ch * bpc) * (NT * R);   // first sample in the channel
  const long long kb = ch * p.Kc + kloc;
  const double4 *pix = p.pix + ch * p.pix_stride;               // this channel's sky records

  double ux[R], uy[R], uz[R], mk[R], mk2[R];
  bool kval[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const long long k = kb + r * NT + tid;
    kval[r] = kloc + r * NT + tid < p.Kc;
    const double4 s = kval[r] ? p.samp[k] : make_double4(0, 0, 0, 0);
    ux[r] = s.x; uy[r] = s.y; uz[r] = s.z;
    const double off = p.use_off ? s.w : 0.0;
    mk[r] = FP64 ? off : kMagic + off;
    mk2[r] = FP64 ? off : kMagic + 0.5 + off;  // odd pixel records: half a turn on
    if (MASKED) s_refs[r][tid] = kval[r] ? p.refs[k] : make_int4(-1, -1, -1, -1);
  }
  unsigned nval_warp = 0;  // valid samples of this warp
#pragma unroll
  for (int r = 0; r < R; ++r) nval_warp += __popc(__ballot_sync(0xffffffffu, kval[r]));

  // accumulators: split -> Kahan FP32 in shared memory; FP64 -> plain double
  double d_re[R], d_im[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    d_re[r] = d_im[r] = 0.0;
    if (!FP64) s_kahan[0][r][tid] = s_kahan[1][r][tid] = s_kahan[2][r][tid] = s_kahan[3][r][tid] = 0.f;
  }

  const int t0 = blockIdx.y * p.tiles_per_chunk;
  const int t1 = min(t0 + p.tiles_per_chunk, p.ntiles);
  constexpr uint32_t kTileBytes = kTilePix * sizeof(double4);

  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();
  if (tid == 0 && t0 < t1) {
    mbar_expect_tx(&s_bar[0], kTileBytes);
    bulk_g2s(s_pix[0], pix + static_cast<long long>(t0) * kTilePix, kTileBytes, &s_bar[0]);
  }

  unsigned long long evaluated = 0, mixed_terms = 0;
  int it = 0;
  for (int t = t0; t < t1; ++t, ++it) {
    const int buf = it & 1;
    const uint32_t par = (it >> 1) & 1;
    if (tid == 0 && t + 1 < t1) {
      mbar_expect_tx(&s_bar[buf ^ 1], kTileBytes);
      bulk_g2s(s_pix[buf ^ 1], pix + static_cast<long long>(t + 1) * kTilePix, kTileBytes,
               &s_bar[buf ^ 1]);
    }
    // classify the tile for this warp's samples
    int mode = 2;
    int st[R];
#pragma unroll
    for (int r = 0; r < R; ++r) st[r] = 2;
    if (MASKED) {
      const double4 cone = p.cones[t];
      bool full = true, any = false;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (kval[r]) {
          st[r] = sample_state(s_refs[r][tid], cone, p.occ);
          full = full && (st[r] == 2);
          any = any || ((st[r] & 3) != 0);
        }
      }
      const bool wfull = __all_sync(0xffffffffu, full);
      const bool wany = __any_sync(0xffffffffu, any);
      mode = wfull ? 2 : (wany ? 1 : 0);
    }
    if (!mbar_wait_bounded(&s_bar[buf], par)) {
      atomicOr(p.err, kErrTimeout);
      s_abort = 1;
    }
    const double4 *tp = s_pix[buf];
    if (mode != 0) {
      if ((tid & 31) == 0) {
        evaluated += static_cast<unsigned long long>(nval_warp) * kTilePix;
        if (mode == 1) mixed_terms += static_cast<unsigned long long>(nval_warp) * kTilePix;
      }
      float t_re[R], t_im[R];
      double e_re[R], e_im[R];
#pragma unroll
      for (int r = 0; r < R; ++r) { t_re[r] = t_im[r] = 0.f; e_re[r] = e_im[r] = 0.0; }
      if (mode == 2) {
        for (int j = 0; j < kTilePix; j += 2) {
          const double4 q0 = tp[j], q1 = tp[j + 1];
          const float I0 = sky_of(q0);
          const float I1 = FP64 ? sky_of(q1) : -sky_of(q1);
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const double t0 = fma(uz[r], q0.z, fma(uy[r], q0.y, fma(ux[r], q0.x, mk[r])));
            fwd_term<FP64>(t0, I0, t_re[r], t_im[r], e_re[r], e_im[r]);
            const double t1 = fma(uz[r], q1.z, fma(uy[r], q1.y, fma(ux[r], q1.x, mk2[r])));
            fwd_term<FP64>(t1, I1, t_re[r], t_im[r], e_re[r], e_im[r]);
          }
        }
      } else {
        // mixed tile: one sample at a time, its occulter rows in registers
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if ((st[r] & 3) == 0) continue;
          if (st[r] == 2) {
            for (int j = 0; j < kTilePix; ++j) {
              const double4 q = tp[j];
              const bool odd = !FP64 && (j & 1);
              const double t = fma(uz[r], q.z, fma(uy[r], q.y, fma(ux[r], q.x, odd ? mk2[r] : mk[r])));
              fwd_term<FP64>(t, odd ? -sky_of(q) : sky_of(q), t_re[r], t_im[r], e_re[r], e_im[r]);
            }
          } else {
            double4 q0, q1, q2;
            mixed_rows(s_refs[r][tid], st[r], p.occ, q0, q1, q2);
            for (int j = 0; j < kTilePix; ++j) {
              const double4 q = tp[j];
              const bool odd = !FP64 && (j & 1);
              float Iv = visible_rows(q0, q1, q2, q.x, q.y, q.z) ? sky_of(q) : 0.f;
              if (odd) Iv = -Iv;
              const double t = fma(uz[r], q.z, fma(uy[r], q.y, fma(ux[r], q.x, odd ? mk2[r] : mk[r])));
              fwd_term<FP64>(t, Iv, t_re[r], t_im[r], e_re[r], e_im[r]);
            }
          }
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (FP64) {
          d_re[r] += e_re[r];
          d_im[r] += e_im[r];
        } else {
          float s0 = s_kahan[0][r][tid], c0 = s_kahan[1][r][tid];
          float s1 = s_kahan[2][r][tid], c1 = s_kahan[3][r][tid];
          kahan_add(s0, c0, t_re[r]);
          kahan_add(s1, c1, t_im[r]);
          s_kahan[0][r][tid] = s0; s_kahan[1][r][tid] = c0;
          s_kahan[2][r][tid] = s1; s_kahan[3][r][tid] = c1;
        }
      }
    }
    __syncthreads();  // every warp is done with buf before it is refilled
    if (s_abort) {
      // a copy was lost: let the other buffer's copy (if any) land, bounded
      if (tid == 0 && t + 1 < t1) mbar_wait_bounded(&s_bar[buf ^ 1], ((it + 1) >> 1) & 1);
      break;
    }
  }

  if (p.counter && (tid & 31) == 0) {
    if (evaluated) atomicAdd(p.counter, evaluated);
    if (mixed_terms) atomicAdd(p.counter + 2, mixed_terms);
  }
  double2 *out = p.part + static_cast<long long>(blockIdx.y) * p.K;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const long long k = kb + r * NT + tid;
    if (!kval[r]) continue;
    double2 v;
    if (FP64) {
      v.x = d_re[r];
      v.y = d_im[r];
    } else {
      v.x = static_cast<double>(s_kahan[0][r][tid]) - static_cast<double>(s_kahan[1][r][tid]);
      v.y = static_cast<double>(s_kahan[2][r][tid]) - static_cast<double>(s_kahan[3][r][tid]);
    }
    out[k] = v;
  }
}

// V_k = sum over chunks (FP64) -> complex64, optionally accumulated.
__global__ void k_reduce_fwd(long long K, int nchunk, const double2 *part, float2 *V,
                             int accumulate) {
  const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double re = 0, im = 0;
  for (int c = 0; c < nchunk; ++c) {
    const double2 v = part[static_cast<long long>(c) * K + k];
    re += v.x;
    im += v.y;
  }
  if (accumulate) {
    const float2 o = V[k];
    re += o.x;
    im += o.y;
  }
  V[k] = make_float2(static_cast<float>(re), static_cast<float>(im));
}

// ======================================================================
// adjoint
// ======================================================================
template <int P, bool MIXED, bool FP64>
__device__ __forceinline__ void adj_sample(const double4 &u, double m, const float2 &a,
                                           const double (&sx)[P], const double (&sy)[P],
                                           const double (&sz)[P], const double4 &q0,
                                           const double4 &q1, const double4 &q2, float (&acc)[P],
                                           double (&dacc)[P]) {
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const double t = fma(u.z, sz[q], fma(u.y, sy[q], fma(u.x, sx[q], m)));
    bool vis = true;
    if (MIXED) vis = visible_rows(q0, q1, q2, sx[q], sy[q], sz[q]);
    if (FP64) {
      double sn, cs;
      sincos_turns_fp64(t, sn, cs);
      const double c = fma(static_cast<double>(a.x), cs, -static_cast<double>(a.y) * sn);
      dacc[q] += vis ? c : 0.0;
    } else {
      float sn, cs;
      sfu_sincos(turn_angle(t), sn, cs);
      if (MIXED) {
        const float ar = vis ? a.x : 0.f, ai = vis ? a.y : 0.f;
        acc[q] = fmaf(ar, cs, acc[q]);
        acc[q] = fmaf(-ai, sn, acc[q]);
      } else {
        acc[q] = fmaf(a.x, cs, acc[q]);
        acc[q] = fmaf(-a.y, sn, acc[q]);
      }
    }
  }
}

template <int NT, int P, int MINB, bool MASKED, bool FP64>
__global__ void __launch_bounds__(NT, MINB) k_adjoint(const AdjParams p) {
  static_assert(P == 4 || P == 8, "a warp covers one or two pixel tiles");
  constexpr int kWarpPix = 32 * P;
  __shared__ float s_kahan[FP64 ? 1 : 2][FP64 ? 1 : P][FP64 ? 1 : NT];  // (sum, comp) per pixel
  __shared__ __align__(128) double4 s_samp[2][kSampTile];
  __shared__ __align__(16) float2 s_coef[2][kSampTile];
  __shared__ __align__(16) int4 s_refs[MASKED ? 2 : 1][MASKED ? kSampTile : 1];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ int s_abort;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kWarps = NT / 32;
  const long long wtile = static_cast<long long>(blockIdx.x) * kWarps + warp;
  const long long pbase = wtile * kWarpPix;
  const bool tile_ok = pbase < p.Jpad;

  double sx[P], sy[P], sz[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const long long j = pbase + q * 32 + lane;
    const double4 v = tile_ok ? p.pix[j] : make_double4(0, 0, 1, 0);
    sx[q] = v.x; sy[q] = v.y; sz[q] = v.z;
  }
  double4 cone0 = make_double4(0, 0, 1, 4.0), cone1 = cone0;
  if (MASKED && tile_ok) {
    cone0 = p.cones[pbase / kTilePix];
    if (P == 8) cone1 = p.cones[pbase / kTilePix + 1];
  }

  double dacc[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    dacc[q] = 0.0;
    if (!FP64) s_kahan[0][q][tid] = s_kahan[1][q][tid] = 0.f;
  }

  // blockIdx.y = channel * nchunk + chunk; a chunk never leaves its channel
  const long long ch = blockIdx.y / p.nchunk;
  const long long k0 = ch * p.Kc + static_cast<long long>(blockIdx.y - ch * p.nchunk) * p.samples_per_chunk;
  const long long k1 = min(k0 + p.samples_per_chunk, (ch + 1) * p.Kc);
  const int ntile = static_cast<int>((k1 - k0 + kSampTile - 1) / kSampTile);

  auto issue = [&](int it, int buf) {
    const long long kk = k0 + static_cast<long long>(it) * kSampTile;
    const int n = static_cast<int>(min(static_cast<long long>(kSampTile), k1 - kk));
    // sizes in multiples of 16 B: samp 32 B each, coef 8 B each (pad to even), refs 16 B
    const int nc = (n + 1) & ~1;
    uint32_t bytes = n * 32u + nc * 8u + (MASKED ? n * 16u : 0u);
    mbar_expect_tx(&s_bar[buf], bytes);
    bulk_g2s(s_samp[buf], p.samp + kk, n * 32u, &s_bar[buf]);
    bulk_g2s(s_coef[buf], p.coef + kk, nc * 8u, &s_bar[buf]);
    if (MASKED) bulk_g2s(s_refs[buf], p.refs + kk, n * 16u, &s_bar[buf]);
  };

  if (tid == 0) {
    mbar_init(&s_bar[0], 1);
    mbar_init(&s_bar[1], 1);
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();
  if (tid == 0 && ntile > 0) issue(0, 0);

  unsigned long long evaluated = 0, mixed_terms = 0;
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  // odd pixel records (odd lanes: record index = pbase + 32 q + lane) are
  // evaluated half a turn on and negated at the end (see the file comment)
  const bool odd_lane = (lane & 1) != 0;
  const double magic = odd_lane ? kMagic + 0.5 : kMagic;
  for (int it = 0; it < ntile; ++it) {
    const int buf = it & 1;
    const uint32_t par = (it >> 1) & 1;
    if (tid == 0 && it + 1 < ntile) issue(it + 1, buf ^ 1);
    if (!mbar_wait_bounded(&s_bar[buf], par)) {
      atomicOr(p.err, kErrTimeout);
      s_abort = 1;
    }
    const long long kk = k0 + static_cast<long long>(it) * kSampTile;
    const int n = static_cast<int>(min(static_cast<long long>(kSampTile), k1 - kk));
    const double4 *sp = s_samp[buf];
    const float2 *cp = s_coef[buf];
    // plain FP32 sums over this staged tile (<= 128 samples per pixel), then
    // one Kahan fold into shared memory
    float t_acc[P];
    double e_acc[P];
#pragma unroll
    for (int q = 0; q < P; ++q) { t_acc[q] = 0.f; e_acc[q] = 0.0; }
    for (int g = 0; g < n; g += 32) {
      // lane l classifies sample g+l against this warp's pixels
      const int gn = min(32, n - g);
      int st = (lane < gn) ? 2 : 0;
      if (MASKED) {
        st = 0;
        if (lane < gn && tile_ok) {
          const int4 rf = s_refs[buf][g + lane];
          st = (P == 8) ? sample_state2(rf, cone0, cone1, p.occ) : sample_state(rf, cone0, p.occ);
        }
      }
      const unsigned live = __ballot_sync(0xffffffffu, (st & 3) != 0);
      const unsigned mixm = __ballot_sync(0xffffffffu, (st & 3) == 1);
      evaluated += static_cast<unsigned long long>(__popc(live)) * kWarpPix;
      mixed_terms += static_cast<unsigned long long>(__popc(mixm)) * kWarpPix;
      // samples visible on every pixel of the warp: no test, uniform loop
      for (unsigned fast = live & ~mixm; fast; fast &= fast - 1) {
        const int i = __ffs(fast) - 1;
        const double4 u = sp[g + i];
        const float2 a = cp[g + i];
        const double uoff = p.use_off ? u.w : 0.0;
        adj_sample<P, false, FP64>(u, FP64 ? uoff : magic + uoff, a, sx, sy, sz, pass, pass,
                                   pass, t_acc, e_acc);
      }
      // samples that need the per-pixel occultation test
      for (unsigned mb = mixm; mb; mb &= mb - 1) {
        const int i = __ffs(mb) - 1;
        const int sst = __shfl_sync(0xffffffffu, st, i);
        const double4 u = sp[g + i];
        const float2 a = cp[g + i];
        const double uoff = p.use_off ? u.w : 0.0;
        double4 q0, q1, q2;
        mixed_rows(s_refs[buf][g + i], sst, p.occ, q0, q1, q2);
        adj_sample<P, true, FP64>(u, FP64 ? uoff : magic + uoff, a, sx, sy, sz, q0, q1, q2,
                                  t_acc, e_acc);
      }
    }
#pragma unroll
    for (int q = 0; q < P; ++q) {
      if (FP64) {
        dacc[q] += e_acc[q];
      } else {
        float s = s_kahan[0][q][tid], c = s_kahan[1][q][tid];
        kahan_add(s, c, t_acc[q]);
        s_kahan[0][q][tid] = s;
        s_kahan[1][q][tid] = c;
      }
    }
    __syncthreads();
    if (s_abort) {
      if (tid == 0 && it + 1 < ntile) mbar_wait_bounded(&s_bar[buf ^ 1], ((it + 1) >> 1) & 1);
      break;
    }
  }

  if (p.counter && lane == 0 && tile_ok) {
    if (evaluated) atomicAdd(p.counter, evaluated);
    if (mixed_terms) atomicAdd(p.counter + 2, mixed_terms);
  }
  if (!tile_ok) return;
  double *out = p.part + static_cast<long long>(blockIdx.y) * p.Jpad;
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const long long j = pbase + q * 32 + lane;
    const double sum =
        FP64 ? dacc[q]
             : static_cast<double>(s_kahan[0][q][tid]) - static_cast<double>(s_kahan[1][q][tid]);
    out[j] = (!FP64 && odd_lane) ? -sum : sum;
  }
}

// image[ch][perm[i]] = scale * sum over the channel's chunks of record i (FP64).
__global__ void k_reduce_adj(long long J, long long Jpad, int nchunk, const double *part,
                             const int *perm, float scale, float *img, int accumulate) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= J) return;
  const long long ch = blockIdx.y;
  part += ch * nchunk * Jpad;
  img += ch * J;
  double s = 0;
  for (int c = 0; c < nchunk; ++c) s += part[static_cast<long long>(c) * Jpad + i];
  s *= static_cast<double>(scale);
  const long long j = perm[i];
  if (accumulate) s += static_cast<double>(img[j]);
  img[j] = static_cast<float>(s);
}

}  // namespace viss

// ---------------------------------------------------------------- launchers
namespace viss {

constexpr int kFwdNT = 256;
constexpr int kAdjNT = 256;

// Launch shapes the plan's tuner chooses among: forward (samples per thread,
// CTAs per SM) and adjoint (pixels per lane, CTAs per SM).
const FwdShape kFwdShapes[kNumFwdShapes] = {{4, 2}, {4, 3}, {2, 3}, {2, 4}};
const AdjShape kAdjShapes[kNumAdjShapes] = {{8, 2}, {8, 3}, {4, 3}, {4, 4}};

template <int R, int MINB, bool M, bool F>
static cudaError_t fwd_inst(const FwdParams &p, int nchunk, cudaStream_t st) {
  const long long per = static_cast<long long>(kFwdNT) * R;
  const long long gx = (p.Kc + per - 1) / per * p.channels;
  if (gx > 0x7fffffffLL) return cudaErrorInvalidValue;
  dim3 grid(static_cast<unsigned>(gx), nchunk);
  k_forward<kFwdNT, R, MINB, M, F><<<grid, kFwdNT, 0, st>>>(p);
  return cudaGetLastError();
}

template <int R, int MINB>
static cudaError_t fwd_m(const FwdParams &p, int nchunk, bool masked, cudaStream_t st) {
  return masked ? fwd_inst<R, MINB, true, false>(p, nchunk, st)
                : fwd_inst<R, MINB, false, false>(p, nchunk, st);
}

cudaError_t launch_forward(const FwdParams &p, int shape, int nchunk, bool masked, bool fp64,
                           cudaStream_t st) {
  if (p.K <= 0 || p.ntiles <= 0) return cudaSuccess;
  if (fp64) return masked ? fwd_inst<2, 1, true, true>(p, nchunk, st) : fwd_inst<2, 1, false, true>(p, nchunk, st);
  switch (shape) {
    case 1: return fwd_m<4, 3>(p, nchunk, masked, st);
    case 2: return fwd_m<2, 3>(p, nchunk, masked, st);
    case 3: return fwd_m<2, 4>(p, nchunk, masked, st);
    default: return fwd_m<4, 2>(p, nchunk, masked, st);
  }
}

int forward_samples_per_block(int shape, bool fp64) {
  if (fp64) return kFwdNT * 2;
  return kFwdNT * kFwdShapes[(shape >= 0 && shape < kNumFwdShapes) ? shape : 0].R;
}
int forward_ctas_per_sm(int shape, bool fp64) {
  if (fp64) return 1;
  return kFwdShapes[(shape >= 0 && shape < kNumFwdShapes) ? shape : 0].minb;
}

cudaError_t launch_reduce_fwd(long long K, int nchunk, const double2 *part, float2 *V, int acc,
                              cudaStream_t st) {
  if (K <= 0) return cudaSuccess;
  k_reduce_fwd<<<static_cast<unsigned>((K + 255) / 256), 256, 0, st>>>(K, nchunk, part, V, acc);
  return cudaGetLastError();
}

int adjoint_pixels_per_block(int shape, bool fp64) {
  if (fp64) return (kAdjNT / 32) * 32 * 4;
  return (kAdjNT / 32) * 32 * kAdjShapes[(shape >= 0 && shape < kNumAdjShapes) ? shape : 0].P;
}
int adjoint_ctas_per_sm(int shape, bool fp64) {
  if (fp64) return 1;
  return kAdjShapes[(shape >= 0 && shape < kNumAdjShapes) ? shape : 0].minb;
}

template <int P, int MINB, bool M, bool F>
static cudaError_t adj_inst(const AdjParams &p, int nchunk, cudaStream_t st) {
  const long long pix_per_cta = static_cast<long long>(kAdjNT / 32) * 32 * P;
  const unsigned gx = static_cast<unsigned>((p.Jpad + pix_per_cta - 1) / pix_per_cta);
  const long long gy = static_cast<long long>(nchunk) * p.channels;
  if (gy > 65535) return cudaErrorInvalidValue;
  dim3 grid(gx, static_cast<unsigned>(gy));
  k_adjoint<kAdjNT, P, MINB, M, F><<<grid, kAdjNT, 0, st>>>(p);
  return cudaGetLastError();
}

template <int P, int MINB>
static cudaError_t adj_m(const AdjParams &p, int nchunk, bool masked, cudaStream_t st) {
  return masked ? adj_inst<P, MINB, true, false>(p, nchunk, st)
                : adj_inst<P, MINB, false, false>(p, nchunk, st);
}

cudaError_t launch_adjoint(const AdjParams &p, int shape, int nchunk, bool masked, bool fp64,
                           cudaStream_t st) {
  if (p.K <= 0 || p.Jpad <= 0) return cudaSuccess;
  if (fp64) return masked ? adj_inst<4, 1, true, true>(p, nchunk, st) : adj_inst<4, 1, false, true>(p, nchunk, st);
  switch (shape) {
    case 1: return adj_m<8, 3>(p, nchunk, masked, st);
    case 2: return adj_m<4, 3>(p, nchunk, masked, st);
    case 3: return adj_m<4, 4>(p, nchunk, masked, st);
    default: return adj_m<8, 2>(p, nchunk, masked, st);
  }
}

cudaError_t launch_reduce_adj(long long J, long long Jpad, int nchunk, int channels,
                              const double *part, const int *perm, float scale, float *img, int acc,
                              cudaStream_t st) {
  if (J <= 0) return cudaSuccess;
  dim3 grid(static_cast<unsigned>((J + 255) / 256), static_cast<unsigned>(channels));
  k_reduce_adj<<<grid, 256, 0, st>>>(J, Jpad, nchunk, part, perm, scale, img, acc);
  return cudaGetLastError();
}

}  // namespace viss
