// healpix.cu -- HEALPix pixel tables on the GPU (FP64).
//
// Replaces pix2ang.cu:61-88 (mk_pix2xy) and pix2ang.cu:92-160
// (f_pix2and_nest).  The reference kernel keeps MATLAB's 1-based table
// indexing (pix2x[ip_low+1], jrll[face_num+1]) and so does not produce HEALPix
// pixel centres; these kernels follow the published HEALPix definition
// (Gorski et al. 2005, ApJ 622:759, sec. 4) whose constants the reference
// tables hold (jrll/jpll, pix2ang.cu:183-184).
//
// Each pixel is reduced to exact integers first -- ring index, pixels per
// quadrant nr, position jp in the ring, the half-pixel shift -- and every
// floating-point quantity is then one or two correctly rounded operations on
// exact integers wherever the formulas allow it:
//   z      = (3N^2 - nr^2)/(3N^2) (caps),  2(2N - i)/(3N) (belt)
//   sin th = sqrt(nr^2 (6N^2 - nr^2) / 9N^4) (caps), sqrt((9N^2-4d^2)/9N^2) (belt)
//   phi    = (2 jp - kshift - 1) pi / (4 nr), with pi as a double-double.
#include "viss_common.cuh"

namespace viss {

__constant__ int c_jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
__constant__ int c_jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

struct PixGeo {
  long long iring, nr, jp, kshift;
  int polar;  // +1 north cap, -1 south cap, 0 belt
};

__device__ __forceinline__ long long isqrt_ll(long long v) {
  long long r = static_cast<long long>(sqrt(static_cast<double>(v)));
  while (r * r > v) --r;
  while ((r + 1) * (r + 1) <= v) ++r;
  return r;
}

__device__ __forceinline__ long long compact_bits(long long v) {
  // keep the even bits of v, packed: 0b..a?b?c -> 0b..abc
  unsigned long long x = static_cast<unsigned long long>(v) & 0x5555555555555555ull;
  x = (x | (x >> 1)) & 0x3333333333333333ull;
  x = (x | (x >> 2)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x >> 4)) & 0x00ff00ff00ff00ffull;
  x = (x | (x >> 8)) & 0x0000ffff0000ffffull;
  x = (x | (x >> 16)) & 0x00000000ffffffffull;
  return static_cast<long long>(x);
}

__device__ __forceinline__ long long spread_bits(long long v) {
  unsigned long long x = static_cast<unsigned long long>(v) & 0x00000000ffffffffull;
  x = (x | (x << 16)) & 0x0000ffff0000ffffull;
  x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
  x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return static_cast<long long>(x);
}

__device__ void ring_geo(long long N, long long p, PixGeo &g) {
  const long long npix = 12 * N * N, ncap = 2 * N * (N - 1);
  if (p < ncap) {
    const long long i = (1 + isqrt_ll(1 + 2 * p)) / 2;
    g.iring = i; g.nr = i; g.jp = p + 1 - 2 * i * (i - 1); g.kshift = 0; g.polar = 1;
  } else if (p < npix - ncap) {
    const long long ip = p - ncap, t = ip / (4 * N);
    g.iring = t + N; g.nr = N; g.jp = ip - 4 * N * t + 1;
    g.kshift = ((g.iring + N) & 1) ? 1 : 0; g.polar = 0;
  } else {
    const long long ip = npix - p, i = (1 + isqrt_ll(2 * ip - 1)) / 2;
    g.iring = 4 * N - i; g.nr = i; g.jp = 4 * i + 1 - (ip - 2 * i * (i - 1));
    g.kshift = 0; g.polar = -1;
  }
}

__device__ void nest_geo(long long N, long long p, PixGeo &g, long long *pix_ix = nullptr,
                         long long *pix_iy = nullptr, int *pix_face = nullptr) {
  const long long npface = N * N;
  const int face = static_cast<int>(p / npface);
  const long long ipf = p - face * npface;
  const long long ix = compact_bits(ipf), iy = compact_bits(ipf >> 1);
  const long long jr = static_cast<long long>(c_jrll[face]) * N - ix - iy - 1;
  long long nr, kshift;
  if (jr < N) { nr = jr; kshift = 0; g.polar = 1; }
  else if (jr > 3 * N) { nr = 4 * N - jr; kshift = 0; g.polar = -1; }
  else { nr = N; kshift = (jr - N) & 1; g.polar = 0; }
  long long jp = (static_cast<long long>(c_jpll[face]) * nr + ix - iy + 1 + kshift) / 2;
  if (jp > 4 * nr) jp -= 4 * nr;
  if (jp < 1) jp += 4 * nr;
  g.iring = jr; g.nr = nr; g.jp = jp; g.kshift = kshift;
  if (pix_ix) { *pix_ix = ix; *pix_iy = iy; *pix_face = face; }
}

__device__ __forceinline__ long long ring_index(long long N, long long iring, long long jp) {
  const long long npix = 12 * N * N, ncap = 2 * N * (N - 1);
  if (iring < N) return 2 * iring * (iring - 1) + jp - 1;
  if (iring <= 3 * N) return ncap + 4 * N * (iring - N) + jp - 1;
  const long long i = 4 * N - iring;
  return npix - 2 * i * (i + 1) + jp - 1;
}

// RING -> NESTED by inverting the NESTED geometry over the 12 faces: on the
// right face ix+iy = jrll*N - ring - 1 and ix-iy = 2 jp - jpll nr - 1 - kshift
// (mod 8 nr); |ix - iy| < N makes the face unique.
__device__ long long ring2nest_one(long long N, long long p) {
  PixGeo g;
  ring_geo(N, p, g);
  const long long mod = 8 * g.nr;
  for (int face = 0; face < 12; ++face) {
    const long long s = static_cast<long long>(c_jrll[face]) * N - g.iring - 1;
    if (s < 0 || s > 2 * N - 2) continue;
    long long d = (2 * g.jp - static_cast<long long>(c_jpll[face]) * g.nr - 1 - g.kshift) % mod;
    if (d > mod / 2) d -= mod;
    if (d <= -mod / 2) d += mod;
    if ((s + d) & 1) continue;
    const long long ix = (s + d) / 2, iy = (s - d) / 2;
    if (ix < 0 || iy < 0 || ix >= N || iy >= N) continue;
    return face * N * N + spread_bits(ix) + (spread_bits(iy) << 1);
  }
  return -1;
}

// ---------------------------------------------------------------- double-double
// Unevaluated sums hi + lo (|lo| <= ulp(hi)/2) built from error-free
// transformations (Dekker / Knuth two-sum, fma two-product).  Used only for
// the pixel tables, to round every output correctly.
struct dd {
  double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
  const double s = __dadd_rn(a, b);
  const double bb = __dadd_rn(s, -a);
  const double e = __dadd_rn(__dadd_rn(a, -__dadd_rn(s, -bb)), __dadd_rn(b, -bb));
  return {s, e};
}
__device__ __forceinline__ dd quick_two_sum(double a, double b) {  // |a| >= |b|
  const double s = __dadd_rn(a, b);
  return {s, __dadd_rn(b, -__dadd_rn(s, -a))};
}
__device__ __forceinline__ dd two_prod(double a, double b) {
  const double p = __dmul_rn(a, b);
  return {p, __fma_rn(a, b, -p)};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  const dd s = two_sum(a.hi, b.hi);
  return quick_two_sum(s.hi, __dadd_rn(s.lo, __dadd_rn(a.lo, b.lo)));
}
__device__ __forceinline__ dd dd_neg(dd a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo = __dadd_rn(p.lo, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
  return quick_two_sum(p.hi, p.lo);
}
__device__ __forceinline__ dd dd_div_d(dd a, double d) {
  const double q1 = __ddiv_rn(a.hi, d);
  const dd p = two_prod(q1, d);
  const double r = __dadd_rn(__dadd_rn(__dadd_rn(a.hi, -p.hi), -p.lo), a.lo);
  return quick_two_sum(q1, __ddiv_rn(r, d));
}
// exact integers a, b (|a|, |b| < 2^53) -> a / b
__device__ __forceinline__ dd dd_ratio(double a, double b) { return dd_div_d({a, 0.0}, b); }
__device__ __forceinline__ dd dd_sqrt(dd a) {
  const double s = __dsqrt_rn(a.hi);
  const dd p = two_prod(s, s);
  const double r = __dadd_rn(__dadd_rn(__dadd_rn(a.hi, -p.hi), -p.lo), a.lo);
  return quick_two_sum(s, __ddiv_rn(r, __dmul_rn(2.0, s)));
}

// pi and pi/2 as double-doubles
__device__ __constant__ double c_pi_hi = 3.141592653589793116, c_pi_lo = 1.2246467991473532e-16;
__device__ __constant__ double c_pio2_hi = 1.5707963267948966, c_pio2_lo = 6.123233995736766e-17;

// sin and cos of a double-double x with |x| <= pi/4 + tiny, by their Taylor
// series (the last term used is below 1e-33).
__device__ void dd_sincos_small(dd x, dd &s, dd &c) {
  const dd x2 = dd_mul(x, x);
  dd ts = x, tc = {1.0, 0.0};
  s = x;
  c = {1.0, 0.0};
  for (int n = 1; n <= 15; ++n) {
    ts = dd_neg(dd_div_d(dd_mul(ts, x2), static_cast<double>((2 * n) * (2 * n + 1))));
    tc = dd_neg(dd_div_d(dd_mul(tc, x2), static_cast<double>((2 * n - 1) * (2 * n))));
    s = dd_add(s, ts);
    c = dd_add(c, tc);
  }
}

// (cos, sin) of k * pi/2 + a from (cos a, sin a): an exact quadrant rotation.
__device__ __forceinline__ void quadrant(long long k, dd ca, dd sa, dd &c, dd &s) {
  switch (static_cast<int>(((k % 4) + 4) % 4)) {
    case 0: c = ca; s = sa; break;
    case 1: c = dd_neg(sa); s = ca; break;
    case 2: c = dd_neg(ca); s = dd_neg(sa); break;
    default: c = sa; s = dd_neg(ca); break;
  }
}

// Angles and unit vector of one pixel centre, every output correctly rounded
// from double-double values: z and sin(theta) are exact rationals (rounded
// once), phi = pi * nphi / den with pi as a double-double, cos/sin(phi) from
// the exact quadrant of nphi/den, and theta = acos(z) corrected by one Newton
// step on cos(theta) - z in double-double.
__device__ void geo_angles(long long N, const PixGeo &g, double &theta, double &phi, double &x,
                           double &y, double &z) {
  const double dN = static_cast<double>(N);
  dd zd, s2;
  if (g.polar != 0) {
    const double nr = static_cast<double>(g.nr);
    const double nr2 = nr * nr;       // exact (nr < 2^26)
    const double d3 = 3.0 * dN * dN;  // exact
    const dd omz = dd_ratio(nr2, d3);                       // 1 - |z|
    const dd zabs = dd_add({1.0, 0.0}, dd_neg(omz));
    zd = g.polar > 0 ? zabs : dd_neg(zabs);
    s2 = dd_mul(omz, dd_ratio(6.0 * dN * dN - nr2, d3));    // sin^2 = omz (2 - omz)
  } else {
    const double d = 2.0 * dN - static_cast<double>(g.iring);  // exact
    zd = dd_ratio(2.0 * d, 3.0 * dN);
    s2 = dd_ratio(9.0 * dN * dN - 4.0 * d * d, 9.0 * dN * dN);
  }
  const dd sth = dd_sqrt(s2);
  z = zd.hi;
  // theta: acos, then one Newton step theta += (cos theta0 - z) / sin theta0
  const double th0 = acos(zd.hi);
  const long long kq = llrint(th0 / c_pio2_hi);
  dd a = two_sum(th0, -static_cast<double>(kq) * c_pio2_hi);
  a = dd_add(a, {-static_cast<double>(kq) * c_pio2_lo, 0.0});
  dd ca, sa, ct, st;
  dd_sincos_small(a, sa, ca);
  quadrant(kq, ca, sa, ct, st);
  const dd resid = dd_add(ct, dd_neg(zd));
  theta = __dadd_rn(th0, __ddiv_rn(resid.hi, st.hi));
  // phi = pi * nphi / den
  const long long nphi = 2 * g.jp - g.kshift - 1, den = 4 * g.nr;
  const dd pn = dd_add(two_prod(static_cast<double>(nphi), c_pi_hi),
                       {__dmul_rn(static_cast<double>(nphi), c_pi_lo), 0.0});
  phi = dd_div_d(pn, static_cast<double>(den)).hi;
  // cos/sin(phi): phi = k pi/2 + r, r = pi (2 nphi - k den) / (2 den), |r| <= pi/4
  const long long kp = (4 * nphi + den) / (2 * den);
  const double m = static_cast<double>(2 * nphi - kp * den);
  const dd r = dd_div_d(dd_add(two_prod(m, c_pi_hi), {__dmul_rn(m, c_pi_lo), 0.0}),
                        2.0 * static_cast<double>(den));
  dd cr, sr, cp, sp;
  dd_sincos_small(r, sr, cr);
  quadrant(kp, cr, sr, cp, sp);
  x = dd_mul(sth, cp).hi;
  y = dd_mul(sth, sp).hi;
}

__global__ void k_mk_pix2xy(int32_t *pix2x, int32_t *pix2y) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 1024) return;
  pix2x[k] = static_cast<int32_t>(compact_bits(k));
  pix2y[k] = static_cast<int32_t>(compact_bits(k >> 1));
}

__global__ void k_pix2ang(long long N, int scheme, long long first, long long count,
                          double *theta, double *phi, double *xyz, int lmn) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  PixGeo g;
  if (scheme == 0) ring_geo(N, first + i, g);
  else nest_geo(N, first + i, g);
  double th, ph, x, y, z;
  geo_angles(N, g, th, ph, x, y, z);
  if (theta) theta[i] = th;
  if (phi) phi[i] = ph;
  if (xyz) {
    xyz[3 * i + 0] = x;
    xyz[3 * i + 1] = lmn ? -y : y;
    xyz[3 * i + 2] = z;
  }
}

__global__ void k_pix_convert(long long N, int from, int to, long long *out) {
  const long long p = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= 12 * N * N) return;
  if (from == to) { out[p] = p; return; }
  if (from == 1) {  // nest -> ring
    PixGeo g;
    nest_geo(N, p, g);
    out[p] = ring_index(N, g.iring, g.jp);
  } else {  // ring -> nest
    out[p] = ring2nest_one(N, p);
  }
}

// healpix_moonback_pre (vissgen3d_blockage.cu:53-74) for FP32 angles: the
// angle edits round to FP32 as the reference stores them; trig in FP64.
__global__ void k_sky_pre(long long n, const float *theta, const float *phi, const float *B,
                          float s, double *lmn, float *Bout) {
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kPi = 3.141592653589793116;
  const float lat = static_cast<float>(kPi / 2 - static_cast<double>(theta[i]));
  float ph = phi[i];
  if (static_cast<double>(ph) > kPi) ph = static_cast<float>(static_cast<double>(ph) - 2 * kPi);
  ph = -ph;
  const double cl = cos(static_cast<double>(lat));
  lmn[3 * i + 0] = cl * cos(static_cast<double>(ph));
  lmn[3 * i + 1] = cl * sin(static_cast<double>(ph));
  lmn[3 * i + 2] = sin(static_cast<double>(lat));
  if (Bout) Bout[i] = __fmul_rn(B[i], s);
}

}  // namespace viss

// ---------------------------------------------------------------- launchers
namespace viss {

cudaError_t launch_mk_pix2xy(int32_t *x, int32_t *y, cudaStream_t st) {
  k_mk_pix2xy<<<4, 256, 0, st>>>(x, y);
  return cudaGetLastError();
}

cudaError_t launch_pix2ang(long long N, int scheme, long long first, long long count,
                           double *theta, double *phi, double *xyz, int lmn, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  k_pix2ang<<<blocks, 256, 0, st>>>(N, scheme, first, count, theta, phi, xyz, lmn);
  return cudaGetLastError();
}

cudaError_t launch_pix_convert(long long N, int from, int to, long long *out, cudaStream_t st) {
  const long long npix = 12 * N * N;
  const unsigned blocks = static_cast<unsigned>((npix + 255) / 256);
  k_pix_convert<<<blocks, 256, 0, st>>>(N, from, to, out);
  return cudaGetLastError();
}

cudaError_t launch_sky_pre(long long n, const float *theta, const float *phi, const float *B,
                           float s, double *lmn, float *Bout, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  k_sky_pre<<<blocks, 256, 0, st>>>(n, theta, phi, B, s, lmn, Bout);
  return cudaGetLastError();
}

}  // namespace viss
