// visibility.cuh -- parameter blocks and launchers of the forward / adjoint
// kernels (visibility.cu), shared with the C ABI layer (capi.cu).
#pragma once

#include "viss_common.cuh"

namespace viss {

constexpr int kSampTile = 128;  // samples per adjoint staging tile
constexpr int kFwdStages = 3;   // shared-memory ring depth: forward pixel tiles
constexpr int kAdjStages = 4;   // shared-memory ring depth: adjoint sample tiles

struct FwdParams {
  const double4 *samp;   // [K] (u, v, w, off)
  const int4 *refs;      // [K] occulter rows or null
  const double4 *occ;    // [G] exact rows
  const float4 *occ32;   // [G] classification rows
  const double4 *pix;    // [Jpad] (l, m, n, sky bits in the low word)
  const float4 *cones;   // [ntiles] tile cones, then [4 * ntiles] sub-tile cones
  long long K;
  int ntiles;
  int tiles_per_chunk;
  double2 *part;                // [nchunk][K]
  unsigned long long *counter;  // [0] exponentials evaluated, [2] of them in mixed tiles
  int *err;
  int use_off;                  // add the per-sample offset (.w) to the phase
  int channels;                 // channel-major sample axis: K = channels * Kc
  long long Kc;                 // samples per channel
  long long pix_stride;         // pixel records per channel's sky (Jpad)
  int drop_tile;                // test hook: CTA (0, 0) skips this tile's copy (-1: none)
};

struct AdjParams {
  const double4 *samp;   // [K] (u, v, w, off)
  const float2 *coef;    // [Kpad] plan-owned copy, padded to an even count
  const int4 *refs;      // [K] or null
  const double4 *occ;    // [G] exact rows
  const float4 *occ32;   // [G] classification rows
  const double4 *pix;    // [Jpad] (l, m, n, -)
  const float4 *cones;   // [ntiles] tile cones, then [4 * ntiles] sub-tile cones
  long long K;
  long long Jpad;         // a multiple of 2 * kTilePix
  int samples_per_chunk;  // multiple of kSampTile
  double *part;           // [nchunk][Jpad]
  unsigned long long *counter;
  int *err;
  int use_off;                  // add the per-sample offset (.w) to the phase
  int channels;                 // one image per channel; K = channels * Kc
  long long Kc;                 // samples per channel (even when channels > 1)
  int nchunk;                   // sample chunks per channel (gridDim.y = channels * nchunk)
  int drop_tile;                // test hook: CTA (0, 0) skips this tile's copy (-1: none)
  // hybrid instance (the occulted gridded adjoint): pairs whose facet the
  // sample sees wholly (facet_open) are skipped, the gridded path takes them
  const float4 *fcones = nullptr;   // [nfacets] facet cones
  long long facet_pix = 0;          // records per facet, a multiple of the warp tile
  long long nfacets = 0;
  // when set: bit (k mod 32) of mixbits[f * mix_words + k / 32] marks the
  // pairs (sample k, facet f) to evaluate (all others skipped unclassified)
  const unsigned *mixbits = nullptr;
  long long mix_words = 0;
};

// Satellite-formation mode (formation.cu): every sample is a pair a < b of the
// S satellites of one snapshot (lexicographic pair order, samples t-major),
// u = U[t][a] - U[t][b].
constexpr int kFormFwdNT = 256;    // forward: threads per block (one snapshot per warp)
constexpr int kFormAdjNT = 256;    // adjoint: threads per block
constexpr int kFormSnapTile = 8;   // snapshots per adjoint staging tile
constexpr int kFormFoldTiles = 32; // forward: pixel tiles between FP64 folds
__host__ __device__ constexpr int form_pairs(int S) { return S * (S - 1) / 2; }
// Adjoint coefficient layout per snapshot: column b (pairs a < b, a = 0..b-1)
// starts at form_col0(b) and is padded to an even length with zeros, so that
// two coefficients load as one 16-byte shared-memory read.
// Columns 1..b-1 hold b' entries each, rounded up to even:
// sum = b(b-1)/2 + (odd b' in [1, b)) = b(b-1)/2 + floor(b/2).
__host__ __device__ constexpr int form_col0(int b) { return b * (b - 1) / 2 + b / 2; }
__host__ __device__ constexpr int form_coef_stride(int S) { return form_col0(S); }

struct FormParams {
  const double4 *U;       // [T][S] satellite vectors in wavelengths (.w unused)
  const double4 *occ;     // exact rows: [T*S] satellites, then [T] snapshots
  const float4 *occ32;    // the same, classification rows
  int sat_rows, snap_rows;  // 1 if those rows are present (and masking is on)
  const double4 *pix;     // forward: pixel + sky records [channel][Jpad]; adjoint: pixel records [Jpad]
  const float4 *cones;    // tile cones (cone_count layout)
  int ntiles;
  long long Jpad;
  long long T;            // snapshots, all channels (channel-major: t = channel * Tc + local)
  long long Tc;           // snapshots per channel
  int channels;
  int tiles_per_chunk;    // forward
  int snaps_per_chunk;    // adjoint, a multiple of kFormSnapTile
  int nchunk;             // forward: chunks; adjoint: chunks per channel
  const float2 *coef;     // adjoint: [T][form_coef_stride(S)] coefficients, offsets applied,
                          // column layout of form_col0
  double2 *part_fwd;      // [chunk][T * B]
  double *part_adj;       // [channel][chunk][Jpad]
  unsigned long long *counter;
  int *err;
};

cudaError_t launch_form_forward(const FormParams &p, int S, int nchunk, cudaStream_t st);
cudaError_t launch_form_adjoint(const FormParams &p, int S, int nchunk, cudaStream_t st);
int form_adjoint_pixels_per_block();

struct FwdShape { int R, minb; };
struct AdjShape { int P, minb; };
constexpr int kNumFwdShapes = 4;
constexpr int kNumAdjShapes = 4;
extern const FwdShape kFwdShapes[kNumFwdShapes];
extern const AdjShape kAdjShapes[kNumAdjShapes];

cudaError_t launch_forward(const FwdParams &p, int shape, int nchunk, bool masked, bool fp64,
                           cudaStream_t st);
int forward_samples_per_block(int shape, bool fp64);
int forward_ctas_per_sm(int shape, bool fp64);
cudaError_t launch_reduce_fwd(long long K, int nchunk, const double2 *part, float2 *V, int acc,
                              cudaStream_t st);
// The occulted split-precision adjoint without the pairs whose facet is
// wholly visible to the sample (p.fcones, p.facet_pix, p.nfacets set).
cudaError_t launch_adjoint_hybrid(const AdjParams &p, int shape, int nchunk, cudaStream_t st);
cudaError_t launch_adjoint(const AdjParams &p, int shape, int nchunk, bool masked, bool fp64,
                           cudaStream_t st);
int adjoint_pixels_per_block(int shape, bool fp64);
int adjoint_ctas_per_sm(int shape, bool fp64);
cudaError_t launch_reduce_adj(long long J, long long Jpad, int nchunk, int channels,
                              const double *part, const int *perm, float scale, float *img, int acc,
                              cudaStream_t st);

}  // namespace viss
