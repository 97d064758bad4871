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
//            through a 3-stage shared-memory ring filled by cp.async.bulk
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
__device__ __forceinline__ int sample_state(const int4 &rf, const float4 &cone,
                                            const float4 *occ32) {
  int st = 2, need = 0;
  const int r3[3] = {rf.x, rf.y, rf.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (r3[c] < 0) continue;
    const int s = cone_state32(cone, occ32[r3[c]]);
    st = min(st, s);
    if (s == 1) need |= 1 << c;
  }
  return st == 1 ? (1 | (need << 2)) : st;
}

// The same against the union of two tiles (a warp tile of 256 pixels): hidden
// only if hidden on both; all visible only if all visible on both; otherwise
// every ref that is not all-visible on both tiles is tested per pixel.
__device__ __forceinline__ int sample_state2(const int4 &rf, const float4 &c0, const float4 &c1,
                                             const float4 *occ32) {
  const int a = sample_state(rf, c0, occ32), b = sample_state(rf, c1, occ32);
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

// The occulter rows a mixed sample must test (need bits 2-4 of its state
// code), compacted to the front: their indices (-1 past the count) and the
// count.
__device__ __forceinline__ int needed_idx(const int4 &rf, int code, int &i0, int &i1, int &i2) {
  i0 = i1 = i2 = -1;
  if (code & 4) i0 = rf.x;
  if (code & 8) {
    if (i0 < 0) i0 = rf.y;
    else i1 = rf.y;
  }
  if (code & 16) {
    if (i0 < 0) i0 = rf.z;
    else if (i1 < 0) i1 = rf.z;
    else i2 = rf.z;
  }
  return (i0 >= 0) + (i1 >= 0) + (i2 >= 0);
}

// Exact rows for those indices; absent rows pass every direction (thr = -4
// is below any dot product of unit vectors).
__device__ __forceinline__ void exact_rows(const double4 *occ, int i0, int i1, int i2,
                                           double4 &q0, double4 &q1, double4 &q2) {
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  q0 = i0 >= 0 ? occ[i0] : pass;
  q1 = i1 >= 0 ? occ[i1] : pass;
  q2 = i2 >= 0 ? occ[i2] : pass;
}

// Classification rows for those indices.
__device__ __forceinline__ void class_rows(const float4 *occ32, int i0, int i1, int i2,
                                           float4 &f0, float4 &f1, float4 &f2) {
  const float4 pass32 = make_float4(0.f, 0.f, 0.f, -4.f);
  f0 = i0 >= 0 ? occ32[i0] : pass32;
  f1 = i1 >= 0 ? occ32[i1] : pass32;
  f2 = i2 >= 0 ? occ32[i2] : pass32;
}

// Both, for one sample; returns how many rows need the test.
__device__ __forceinline__ int needed_rows(const int4 &rf, int code, const double4 *occ,
                                           const float4 *occ32, double4 &q0, double4 &q1,
                                           double4 &q2, float4 &f0, float4 &f1, float4 &f2) {
  int i0, i1, i2;
  const int n = needed_idx(rf, code, i0, i1, i2);
  exact_rows(occ, i0, i1, i2, q0, q1, q2);
  class_rows(occ32, i0, i1, i2, f0, f1, f2);
  return n;
}

// State of one cone against the first n classification rows (2 visible, 0
// hidden, 1 mixed).
__device__ __forceinline__ int rows_state(const float4 &cone, int n, const float4 &f0,
                                          const float4 &f1, const float4 &f2) {
  int st = 2;
  if (n > 0) st = min(st, cone_state32(cone, f0));
  if (n > 1) st = min(st, cone_state32(cone, f1));
  if (n > 2) st = min(st, cone_state32(cone, f2));
  return st;
}

// Exact visibility of direction s against the first NROWS rows (the same IEEE
// operations as the CPU oracle's predicate).
template <int NROWS>
__device__ __forceinline__ bool visible_rows(const double4 &q0, const double4 &q1,
                                             const double4 &q2, double s0, double s1, double s2) {
  bool v = true;
  if (NROWS > 0) v = dot_exact(s0, s1, s2, q0) >= q0.w;
  if (NROWS > 1) v = v & (dot_exact(s0, s1, s2, q1) >= q1.w);
  if (NROWS > 2) v = v & (dot_exact(s0, s1, s2, q2) >= q2.w);
  return v;
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
// Pixels per forward sub-tile (the span a mixed sample row is refined to).
constexpr int kSubPix = 32;

// One sample over kSubPix staged records, in pairs (even record at mk, odd
// record half a turn on at mk2 and negated), testing the first NROWS
// occulter rows per term (NROWS = 0: every pixel visible).
template <int NROWS, bool FP64>
__device__ __forceinline__ void fwd_span(const double4 *tp, double ux, double uy, double uz,
                                         double mk, double mk2, const double4 &q0,
                                         const double4 &q1, const double4 &q2, float &re,
                                         float &im, double &dre, double &dim) {
#pragma unroll 2
  for (int j = 0; j < kSubPix; j += 2) {
    const double4 a = tp[j], b = tp[j + 1];
    float Ia = sky_of(a), Ib = FP64 ? sky_of(b) : -sky_of(b);
    if (NROWS > 0) {
      Ia = visible_rows<NROWS>(q0, q1, q2, a.x, a.y, a.z) ? Ia : 0.f;
      Ib = visible_rows<NROWS>(q0, q1, q2, b.x, b.y, b.z) ? Ib : 0.f;
    }
    const double ta = fma(uz, a.z, fma(uy, a.y, fma(ux, a.x, mk)));
    fwd_term<FP64>(ta, Ia, re, im, dre, dim);
    const double tb = fma(uz, b.z, fma(uy, b.y, fma(ux, b.x, mk2)));
    fwd_term<FP64>(tb, Ib, re, im, dre, dim);
  }
}

template <int NT, int R, int MINB, bool MASKED, bool FP64>
__global__ void __launch_bounds__(NT, MINB) k_forward(const FwdParams p) {
  constexpr int S = kFwdStages;
  constexpr int kWarps = NT / 32;
  __shared__ __align__(128) double4 s_pix[S][kTilePix];
  __shared__ __align__(16) int4 s_refs[MASKED ? R : 1][MASKED ? NT : 1];
  // Kahan (sum, comp) of re and im per sample, kept in shared memory (touched
  // once per tile) so the registers hold only what the inner loop needs
  __shared__ float s_kahan[FP64 ? 1 : 4][FP64 ? 1 : R][FP64 ? 1 : NT];
  __shared__ __align__(8) uint64_t s_full[S], s_empty[S];
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;

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
  const int ntile = max(0, min(t0 + p.tiles_per_chunk, p.ntiles) - t0);
  constexpr uint32_t kTileBytes = kTilePix * sizeof(double4);
  // test hook (viss_plan_debug_drop_copy): the first CTA never stages one
  // tile, so its bounded waits run out and the error flag is raised
  const int drop = (blockIdx.x == 0 && blockIdx.y == 0) ? p.drop_tile : -1;
  auto issue = [&](int i, int stage) {
    if (i == drop) return;
    mbar_expect_tx(&s_full[stage], kTileBytes);
    bulk_g2s(s_pix[stage], pix + static_cast<long long>(t0 + i) * kTilePix, kTileBytes,
             &s_full[stage]);
  };

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mbar_init(&s_full[s], 1);
      mbar_init(&s_empty[s], kWarps);
    }
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();

  unsigned long long evaluated = 0, mixed_terms = 0;
  unsigned sup = 0;  // per-row super-tile states (MASKED)
  int next = 0;  // next tile to issue (producer state, thread 0)
  for (int it = 0; it < ntile; ++it) {
    const int t = t0 + it, stage = it % S;
    if (tid == 0 && !ring_refill<S>(s_empty, next, it, ntile, issue)) {
      atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
    }
    if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
    // classify the tile for this warp's samples
    int mode = 2;
    int st[R];
#pragma unroll
    for (int r = 0; r < R; ++r) st[r] = 2;
    if (MASKED) {
      // once per super-tile: samples wholly visible (2) or wholly hidden (0)
      // there skip the per-tile test; 1 = test each tile (2 bits per row)
      if (it == 0 || (t & (kSuperTiles - 1)) == 0) {
        const float4 sc = p.cones[5LL * p.ntiles + t / kSuperTiles];
        sup = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int s = kval[r] ? (sample_state(s_refs[r][tid], sc, p.occ32) & 3) : 2;
          sup |= static_cast<unsigned>(s) << (2 * r);
        }
      }
      const float4 cone = p.cones[t];
      bool full = true, any = false;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if (kval[r]) {
          const unsigned known = (sup >> (2 * r)) & 3u;
          st[r] = known != 1 ? static_cast<int>(known) : sample_state(s_refs[r][tid], cone, p.occ32);
          full = full && (st[r] == 2);
          any = any || ((st[r] & 3) != 0);
        }
      }
      const bool wfull = __all_sync(0xffffffffu, full);
      const bool wany = __any_sync(0xffffffffu, any);
      mode = wfull ? 2 : (wany ? 1 : 0);
    }
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_full[stage], static_cast<uint32_t>(it / S) & 1u))) {
      if ((tid & 31) == 0) atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
      break;
    }
    const double4 *tp = s_pix[stage];
    if (mode != 0) {
      float t_re[R], t_im[R];
      double e_re[R], e_im[R];
#pragma unroll
      for (int r = 0; r < R; ++r) { t_re[r] = t_im[r] = 0.f; e_re[r] = e_im[r] = 0.0; }
      if (mode == 2) {
        if ((tid & 31) == 0) evaluated += static_cast<unsigned long long>(nval_warp) * kTilePix;
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
        // mixed tile: one sample row at a time.  A lane whose sample needs
        // the per-term test classifies it against the tile's four 32-pixel
        // sub-tile cones; the warp then runs each sub-tile once, with the
        // exact test of as many occulter rows as its neediest lane has there
        // (lanes that see all of the sub-tile pass every test by
        // construction), or without a test, and skips a sub-tile no lane
        // sees.  Lanes that see none of a sub-tile sit it out.
        const float4 *sub = p.cones + p.ntiles + 4LL * t;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int code = kval[r] ? st[r] : 0;
          double4 q0, q1, q2;
          float4 f0, f1, f2;
          const int nr = needed_rows(s_refs[r][tid], (code & 3) == 1 ? code : 0, p.occ, p.occ32,
                                     q0, q1, q2, f0, f1, f2);
          // 2 bits per sub-tile: 2 all visible, 0 none, 1 test per pixel
          unsigned ss = (code & 3) == 2 ? 0xAAu : 0u;
          if ((code & 3) == 1) {
#pragma unroll
            for (int b = 0; b < 4; ++b) ss |= static_cast<unsigned>(rows_state(sub[b], nr, f0, f1, f2)) << (2 * b);
          }
#pragma unroll 1
          for (int b = 0; b < 4; ++b) {
            const unsigned sst = (ss >> (2 * b)) & 3u;
            const unsigned seen = __ballot_sync(0xffffffffu, sst != 0);
            if (seen == 0) continue;
            const int wn = __reduce_max_sync(0xffffffffu, sst == 1 ? nr : 0);
            if ((tid & 31) == 0) {
              evaluated += static_cast<unsigned long long>(__popc(seen)) * kSubPix;
              if (wn) mixed_terms += static_cast<unsigned long long>(__popc(seen)) * kSubPix;
            }
            if (sst == 0) continue;
            const double4 *sp = tp + b * kSubPix;
            if (wn == 0)
              fwd_span<0, FP64>(sp, ux[r], uy[r], uz[r], mk[r], mk2[r], q0, q1, q2, t_re[r], t_im[r], e_re[r], e_im[r]);
            else if (wn == 1)
              fwd_span<1, FP64>(sp, ux[r], uy[r], uz[r], mk[r], mk2[r], q0, q1, q2, t_re[r], t_im[r], e_re[r], e_im[r]);
            else if (wn == 2)
              fwd_span<2, FP64>(sp, ux[r], uy[r], uz[r], mk[r], mk2[r], q0, q1, q2, t_re[r], t_im[r], e_re[r], e_im[r]);
            else
              fwd_span<3, FP64>(sp, ux[r], uy[r], uz[r], mk[r], mk2[r], q0, q1, q2, t_re[r], t_im[r], e_re[r], e_im[r]);
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
    ring_release(s_empty, stage);
  }
  if (tid == 0) ring_drain<S>(s_full, next);

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
// One sample into a lane's P pixels (pixel q of every lane lies in the warp's
// 32-pixel sub-tile q).  Bit q of the warp-uniform `hid` zeroes sub-tile q
// (none of it visible); NROWS > 0 tests the first NROWS occulter rows on
// every term.  The P terms stay one branch-free block: splitting them by
// sub-tile would serialise their DFMA -> MUFU latency chains, which costs more
// than evaluating a hidden term.
template <int P, int NROWS, bool FP64>
__device__ __forceinline__ void adj_sample(const double4 &u, double m, const float2 &a,
                                           const double (&sx)[P], const double (&sy)[P],
                                           const double (&sz)[P], const double4 &q0,
                                           const double4 &q1, const double4 &q2, unsigned hid,
                                           float (&acc)[P], double (&dacc)[P]) {
#pragma unroll
  for (int q = 0; q < P; ++q) {
    const double t = fma(u.z, sz[q], fma(u.y, sy[q], fma(u.x, sx[q], m)));
    bool vis = ((hid >> q) & 1u) == 0;
    if (NROWS > 0) vis = vis & visible_rows<NROWS>(q0, q1, q2, sx[q], sy[q], sz[q]);
    const float ar = vis ? a.x : 0.f, ai = vis ? a.y : 0.f;
    if (FP64) {
      double sn, cs;
      sincos_turns_fp64(t, sn, cs);
      dacc[q] += fma(static_cast<double>(ar), cs, -static_cast<double>(ai) * sn);
    } else {
      float sn, cs;
      sfu_sincos(turn_angle(t), sn, cs);
      acc[q] = fmaf(ar, cs, acc[q]);
      acc[q] = fmaf(-ai, sn, acc[q]);
    }
  }
}

template <int NT, int P, int MINB, bool MASKED, bool FP64, bool HYBRID = false>
__global__ void __launch_bounds__(NT, MINB) k_adjoint(const AdjParams p) {
  static_assert(P == 4 || P == 8, "a warp covers one or two pixel tiles");
  constexpr int kWarpPix = 32 * P;
  __shared__ float s_kahan[FP64 ? 1 : 2][FP64 ? 1 : P][FP64 ? 1 : NT];  // (sum, comp) per pixel
  constexpr int S = kAdjStages;
  __shared__ __align__(128) double4 s_samp[S][kSampTile];
  __shared__ __align__(16) float2 s_coef[S][kSampTile];
  __shared__ __align__(16) int4 s_refs[MASKED ? S : 1][MASKED ? kSampTile : 1];
  __shared__ __align__(8) uint64_t s_full[S], s_empty[S];
  __shared__ int s_abort;
  volatile int *abort_flag = &s_abort;
  constexpr int kWarps = NT / 32;
  // each warp's P sub-tile cones (sub-tile q = pixels pbase + 32 q .. + 31)
  __shared__ float4 s_sub[MASKED ? kWarps : 1][MASKED ? P : 1];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
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
  // the warp's tile cone(s) in registers, its sub-tile cones in shared memory
  float4 cone0 = make_float4(0.f, 0.f, 1.f, 4.f), cone1 = cone0;
  float4 fcone = cone0;   // hybrid: the cone of the facet holding this warp's pixels
  if (MASKED && tile_ok) {
    const long long ntiles = p.Jpad / kTilePix;
    cone0 = p.cones[pbase / kTilePix];
    if (P == 8) cone1 = p.cones[pbase / kTilePix + 1];
    if (lane < P) s_sub[warp][lane] = p.cones[ntiles + pbase / 32 + lane];
    if (HYBRID) fcone = p.fcones[min(pbase / p.facet_pix, p.nfacets - 1)];
  }
  // hybrid with the mixed-pair bitmask: this warp's facet row of it
  const unsigned *mixrow =
      (HYBRID && p.mixbits) ? p.mixbits + min(pbase / max(p.facet_pix, 1LL), p.nfacets - 1) * p.mix_words : nullptr;
  __syncwarp();

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

  // test hook (viss_plan_debug_drop_copy), as in the forward
  const int drop = (blockIdx.x == 0 && blockIdx.y == 0) ? p.drop_tile : -1;
  auto issue = [&](int i, int stage) {
    if (i == drop) return;
    const long long kk = k0 + static_cast<long long>(i) * kSampTile;
    const int n = static_cast<int>(min(static_cast<long long>(kSampTile), k1 - kk));
    // sizes in multiples of 16 B: samp 32 B each, coef 8 B each (pad to even), refs 16 B
    const int nc = (n + 1) & ~1;
    uint32_t bytes = n * 32u + nc * 8u + (MASKED ? n * 16u : 0u);
    mbar_expect_tx(&s_full[stage], bytes);
    bulk_g2s(s_samp[stage], p.samp + kk, n * 32u, &s_full[stage]);
    bulk_g2s(s_coef[stage], p.coef + kk, nc * 8u, &s_full[stage]);
    if (MASKED) bulk_g2s(s_refs[stage], p.refs + kk, n * 16u, &s_full[stage]);
  };

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
      mbar_init(&s_full[s], 1);
      mbar_init(&s_empty[s], kWarps);
    }
    fence_mbar_init();
    s_abort = 0;
  }
  __syncthreads();
  int next = 0;  // next tile to issue (producer state, thread 0)

  unsigned long long evaluated = 0, mixed_terms = 0;
  const double4 pass = make_double4(0.0, 0.0, 0.0, -4.0);
  // odd pixel records (odd lanes: record index = pbase + 32 q + lane) are
  // evaluated half a turn on and negated at the end (see the file comment)
  const bool odd_lane = (lane & 1) != 0;
  const double magic = odd_lane ? kMagic + 0.5 : kMagic;
  for (int it = 0; it < ntile; ++it) {
    const int buf = it % S;
    if (tid == 0 && !ring_refill<S>(s_empty, next, it, ntile, issue)) {
      atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
    }
    if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
    if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_full[buf], static_cast<uint32_t>(it / S) & 1u))) {
      if (lane == 0) atomicOr(p.err, kErrTimeout);
      *abort_flag = 1;
      break;
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
      // lane l classifies sample g+l against this warp's pixels; a sample
      // that is mixed on the warp's tile(s) is refined against the P
      // sub-tile cones: subm = hidden sub-tiles (bits 0-7) | sub-tiles that
      // need the per-pixel test (bits 8-15)
      const int gn = min(32, n - g);
      int st = (lane < gn) ? 2 : 0;
      unsigned subm = 0;
      if (MASKED) {
        st = 0;
        // hybrid: a sample that sees the whole facet is the gridded path's,
        // one hidden on all of it contributes nothing; with the bitmask both
        // are skipped without loading their rows (kk + g is a multiple of 32)
        const bool skip_pair =
            HYBRID && mixrow && !((__ldg(mixrow + (kk + g) / 32) >> lane) & 1u);
        if (lane < gn && tile_ok && !skip_pair) {
          const int4 rf = s_refs[buf][g + lane];
          st = (HYBRID && !mixrow && facet_open(rf, fcone, p.occ32))
                   ? 0
                   : ((P == 8) ? sample_state2(rf, cone0, cone1, p.occ32) : sample_state(rf, cone0, p.occ32));
          if ((st & 3) == 1) {
            int i0, i1, i2;
            const int nr = needed_idx(rf, st, i0, i1, i2);
            float4 f0, f1, f2;
            class_rows(p.occ32, i0, i1, i2, f0, f1, f2);
            unsigned hid = 0, mix = 0;
#pragma unroll
            for (int q = 0; q < P; ++q) {
              const int ss = rows_state(s_sub[warp][q], nr, f0, f1, f2);
              hid |= static_cast<unsigned>(ss == 0) << q;
              mix |= static_cast<unsigned>(ss == 1) << q;
            }
            if (hid == (1u << P) - 1) st = 0;  // hidden on every sub-tile
            subm = hid | (mix << 8);
          }
        }
      }
      const unsigned live = __ballot_sync(0xffffffffu, (st & 3) != 0);
      const unsigned mixm = __ballot_sync(0xffffffffu, (st & 3) == 1);
      evaluated += static_cast<unsigned long long>(__popc(live)) * kWarpPix;
      if (MASKED && mixm)  // samples that run the per-term test, on all their P sub-tiles
        mixed_terms += static_cast<unsigned long long>(
                           __popc(__ballot_sync(0xffffffffu, (st & 3) == 1 && (subm >> 8) != 0))) *
                       kWarpPix;
      // samples visible on every pixel of the warp: no test, uniform loop
      for (unsigned fast = live & ~mixm; fast; fast &= fast - 1) {
        const int i = __ffs(fast) - 1;
        const double4 u = sp[g + i];
        const float2 a = cp[g + i];
        const double uoff = p.use_off ? u.w : 0.0;
        adj_sample<P, 0, FP64>(u, FP64 ? uoff : magic + uoff, a, sx, sy, sz, pass, pass, pass,
                               0u, t_acc, e_acc);
      }
      // samples mixed on the warp's tiles: hidden sub-tiles zeroed; the exact
      // per-term test only for samples with a sub-tile that needs it
      for (unsigned mb = mixm; mb; mb &= mb - 1) {
        const int i = __ffs(mb) - 1;
        const unsigned sm = __shfl_sync(0xffffffffu, subm, i);
        const unsigned hid = sm & 0xffu;
        const double4 u = sp[g + i];
        const float2 a = cp[g + i];
        const double uoff = p.use_off ? u.w : 0.0;
        const double mm = FP64 ? uoff : magic + uoff;
        if ((sm >> 8) == 0) {
          adj_sample<P, 0, FP64>(u, mm, a, sx, sy, sz, pass, pass, pass, hid, t_acc, e_acc);
          continue;
        }
        const int sst = __shfl_sync(0xffffffffu, st, i);
        int i0, i1, i2;
        const int nr = needed_idx(s_refs[buf][g + i], sst, i0, i1, i2);
        double4 q0, q1, q2;
        exact_rows(p.occ, i0, i1, i2, q0, q1, q2);
        if (nr == 1)
          adj_sample<P, 1, FP64>(u, mm, a, sx, sy, sz, q0, q1, q2, hid, t_acc, e_acc);
        else if (nr == 2)
          adj_sample<P, 2, FP64>(u, mm, a, sx, sy, sz, q0, q1, q2, hid, t_acc, e_acc);
        else
          adj_sample<P, 3, FP64>(u, mm, a, sx, sy, sz, q0, q1, q2, hid, t_acc, e_acc);
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
    ring_release(s_empty, buf);
  }
  if (tid == 0) ring_drain<S>(s_full, next);

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
constexpr int kAdjNT = 128;  // 4 warps: less coupling of uneven warps through the ring

// Launch shapes the plan's tuner chooses among: forward (samples per thread,
// CTAs per SM) and adjoint (pixels per lane, CTAs per SM).
const FwdShape kFwdShapes[kNumFwdShapes] = {{4, 2}, {4, 3}, {2, 3}, {2, 4}};
const AdjShape kAdjShapes[kNumAdjShapes] = {{8, 4}, {8, 5}, {4, 5}, {4, 6}};

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

template <int P, int MINB, bool M, bool F, bool H = false>
static cudaError_t adj_inst(const AdjParams &p, int nchunk, cudaStream_t st) {
  const long long pix_per_cta = static_cast<long long>(kAdjNT / 32) * 32 * P;
  const unsigned gx = static_cast<unsigned>((p.Jpad + pix_per_cta - 1) / pix_per_cta);
  const long long gy = static_cast<long long>(nchunk) * p.channels;
  if (gy > 65535) return cudaErrorInvalidValue;
  dim3 grid(gx, static_cast<unsigned>(gy));
  k_adjoint<kAdjNT, P, MINB, M, F, H><<<grid, kAdjNT, 0, st>>>(p);
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
    case 1: return adj_m<8, 5>(p, nchunk, masked, st);
    case 2: return adj_m<4, 5>(p, nchunk, masked, st);
    case 3: return adj_m<4, 6>(p, nchunk, masked, st);
    default: return adj_m<8, 4>(p, nchunk, masked, st);
  }
}

cudaError_t launch_adjoint_hybrid(const AdjParams &p, int shape, int nchunk, cudaStream_t st) {
  if (p.K <= 0 || p.Jpad <= 0) return cudaSuccess;
  // a facet must hold whole warp tiles of the widest shape (32 lanes x 8 pixels)
  if (!p.fcones || p.facet_pix <= 0 || p.facet_pix % (32 * 8) != 0 || p.nfacets <= 0 || !p.refs)
    return cudaErrorInvalidValue;
  switch (shape) {
    case 1: return adj_inst<8, 5, true, false, true>(p, nchunk, st);
    case 2: return adj_inst<4, 5, true, false, true>(p, nchunk, st);
    case 3: return adj_inst<4, 6, true, false, true>(p, nchunk, st);
    default: return adj_inst<8, 4, true, false, true>(p, nchunk, st);
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
