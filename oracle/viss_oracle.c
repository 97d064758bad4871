/*
 * viss_oracle.c -- CPU restatement of the viss_optimize_3d hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA library's results are tested against it:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it.  Nothing in the product (viss_optimize_3d_b200/, the C ABI, the host
 * executables) links or calls it.
 *
 * Every function restates one piece of the reference program
 * (SSshuishui/viss_optimize_3d) in FP64 (long double where it pays), with the
 * file:line it follows.  Reference files are CUDA kernels with no CPU path,
 * so this is a port of their arithmetic, not a call into them:
 *
 *   HEALPix pix2ang (RING and NESTED)   pix2ang.cu:61-160 (mk_pix2xy,
 *       f_pix2and_nest).  pix2ang.cu keeps MATLAB 1-based table indexing and
 *       does not reproduce HEALPix; this oracle follows the published HEALPix
 *       definition (Gorski et al. 2005, ApJ 622:759, sec. 4) that the
 *       reference's tables (jrll/jpll at pix2ang.cu:183-184) come from.
 *   sky direction convention            vissgen3d_blockage.cu:53-74
 *   occultation predicate               vissgen3d_blockage.cu:88-94,180-186,
 *                                        constants :249-252
 *   forward visibilities                vissgen3d_blockage.cu:76-102
 *   shell histogram + DCF               vissgen3d_blockage.cu:105-130,
 *                                        vissgen3d_noblockage.cu:132-141
 *   w-rotation and elevation factor     vissgen3d_blockage.cu:144-164
 *   imaging adjoint                     vissgen3d_blockage.cu:167-192
 *
 * Build: gcc -O2 -ffp-contract=off -fopenmp -shared -fPIC (oracle/Makefile).
 * -ffp-contract=off matters: the occultation predicate is defined with an
 * explicit fma() order so that CPU and GPU evaluate the same IEEE operations.
 */
#define _GNU_SOURCE
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI_L 3.141592653589793238462643383279502884L

/* ------------------------------------------------------------------------ */
/* HEALPix                                                                   */
/* ------------------------------------------------------------------------ */

/* Face layout of the 12 base pixels: ring-row (in units of nside) and
 * longitude offset (in units of pi/4).  Published HEALPix constants, the same
 * numbers as pix2ang.cu:183-184. */
static const int orc_jrll[12] = {2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4};
static const int orc_jpll[12] = {1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7};

/* pix2ang.cu:61-88 (mk_pix2xy): split the bits of a 10-bit in-face index into
 * x (even bits) and y (odd bits). */
void orc_mk_pix2xy(int32_t *pix2x, int32_t *pix2y)
{
    for (int k = 0; k < 1024; ++k) {
        int x = 0, y = 0;
        for (int b = 0; b < 5; ++b) {
            x |= ((k >> (2 * b)) & 1) << b;
            y |= ((k >> (2 * b + 1)) & 1) << b;
        }
        pix2x[k] = x;
        pix2y[k] = y;
    }
}

static int64_t orc_compact_bits(int64_t v)
{
    int64_t r = 0;
    for (int b = 0; b < 31; ++b) r |= ((v >> (2 * b)) & 1) << b;
    return r;
}

static int64_t orc_spread_bits(int64_t v)
{
    int64_t r = 0;
    for (int b = 0; b < 31; ++b) r |= ((v >> b) & 1) << (2 * b);
    return r;
}

static int64_t orc_isqrt(int64_t v)
{
    int64_t r = (int64_t)sqrt((double)v);
    while (r * r > v) --r;
    while ((r + 1) * (r + 1) <= v) ++r;
    return r;
}

/* Geometry of one pixel centre, exact integers plus the rational pieces:
 *   ring index i in [1, 4N-1], nr = pixels-per-quarter of the ring,
 *   z = cos(theta), with 1-|z| kept separately for the polar caps,
 *   phi/pi = (2*jp - kshift - 1) / (4*nr)   (jp in [1, 4nr]). */
typedef struct {
    int64_t iring, nr, jp, kshift;
    int polar;       /* +1 north cap, -1 south cap, 0 equatorial belt */
} orc_pixgeo;

static void orc_ring_geo(int64_t nside, int64_t p, orc_pixgeo *g)
{
    const int64_t npix = 12 * nside * nside;
    const int64_t ncap = 2 * nside * (nside - 1);
    if (p < ncap) {
        int64_t i = (1 + orc_isqrt(1 + 2 * p)) / 2;
        g->iring = i;
        g->nr = i;
        g->jp = p + 1 - 2 * i * (i - 1);
        g->kshift = 0;
        g->polar = 1;
    } else if (p < npix - ncap) {
        int64_t ip = p - ncap;
        int64_t t = ip / (4 * nside);
        g->iring = t + nside;
        g->nr = nside;
        g->jp = ip - 4 * nside * t + 1;
        g->kshift = ((g->iring + nside) & 1) ? 1 : 0;
        g->polar = 0;
    } else {
        int64_t ip = npix - p;
        int64_t i = (1 + orc_isqrt(2 * ip - 1)) / 2;
        g->iring = 4 * nside - i;
        g->nr = i;
        g->jp = 4 * i + 1 - (ip - 2 * i * (i - 1));
        g->kshift = 0;
        g->polar = -1;
    }
}

static void orc_nest_geo(int64_t nside, int64_t p, orc_pixgeo *g)
{
    const int64_t npface = nside * nside;
    const int face = (int)(p / npface);
    const int64_t ipf = p % npface;
    const int64_t ix = orc_compact_bits(ipf);
    const int64_t iy = orc_compact_bits(ipf >> 1);
    const int64_t jr = (int64_t)orc_jrll[face] * nside - ix - iy - 1;
    int64_t nr, kshift;
    if (jr < nside) {
        nr = jr; kshift = 0; g->polar = 1;
    } else if (jr > 3 * nside) {
        nr = 4 * nside - jr; kshift = 0; g->polar = -1;
    } else {
        nr = nside; kshift = (jr - nside) & 1; g->polar = 0;
    }
    int64_t jp = ((int64_t)orc_jpll[face] * nr + ix - iy + 1 + kshift) / 2;
    if (jp > 4 * nr) jp -= 4 * nr;
    if (jp < 1) jp += 4 * nr;
    g->iring = jr;
    g->nr = nr;
    g->jp = jp;
    g->kshift = kshift;
}

/* Angles and unit vector of one pixel centre in quad precision (113-bit
 * significand), so that rounding to double is the correctly rounded value
 * (double rounding is then astronomically unlikely).  cos(phi) and sin(phi)
 * are exactly zero where phi is a multiple of pi/2. */
static void orc_geo_angles(int64_t nside, const orc_pixgeo *g, __float128 *theta,
                           __float128 *phi, __float128 v[3])
{
    const __float128 N = (__float128)nside;
    __float128 z, sth;
    if (g->polar != 0) {
        /* 1 - |z| = nr^2 / (3 N^2): exact rational, no cancellation */
        __float128 omz = ((__float128)g->nr * (__float128)g->nr) / (3 * N * N);
        sth = sqrtq(omz * (2 - omz));
        z = (g->polar > 0) ? 1 - omz : omz - 1;
        __float128 half = 2 * asinq(sqrtq(omz / 2));      /* angle from the pole */
        *theta = (g->polar > 0) ? half : M_PIq - half;
    } else {
        z = (2 * N - (__float128)g->iring) * 2 / (3 * N);
        sth = sqrtq((1 - z) * (1 + z));
        *theta = acosq(z);
    }
    const int64_t num = 2 * g->jp - g->kshift - 1, den = 4 * g->nr;   /* phi = pi num/den */
    *phi = M_PIq * (__float128)num / (__float128)den;
    __float128 c = cosq(*phi), sn = sinq(*phi);
    if ((2 * num) % den == 0 && ((2 * num / den) & 1)) c = 0;        /* phi = pi/2 + k pi */
    if (num % den == 0) sn = 0;                                      /* phi = k pi */
    v[0] = sth * c;
    v[1] = sth * sn;
    v[2] = z;
}

/* pix2ang.cu:92-160 (f_pix2and_nest) and its RING counterpart: theta, phi
 * and the HEALPix unit vector (x, y, z) of pixels [first, first+count).
 * scheme 0 = RING, 1 = NESTED.  Any output pointer may be NULL.
 * Returns 0, or -1 for a bad nside / range. */
int orc_pix2ang(int nside, int scheme, int64_t first, int64_t count, double *theta,
                double *phi, double *xyz)
{
    if (nside < 1 || nside > (1 << 29)) return -1;
    const int64_t npix = 12LL * nside * nside;
    if (first < 0 || count < 0 || first + count > npix) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
        orc_pixgeo g;
        if (scheme == 0) orc_ring_geo(nside, first + i, &g);
        else orc_nest_geo(nside, first + i, &g);
        __float128 th, ph, v[3];
        orc_geo_angles(nside, &g, &th, &ph, v);
        if (theta) theta[i] = (double)th;
        if (phi) phi[i] = (double)ph;
        if (xyz) {
            xyz[3 * i + 0] = (double)v[0];
            xyz[3 * i + 1] = (double)v[1];
            xyz[3 * i + 2] = (double)v[2];
        }
    }
    return 0;
}

/* Ring index / pixel-in-ring of a pixel, both schemes (exact integers). */
int orc_pix2ring(int nside, int scheme, int64_t p, int64_t *iring, int64_t *jp)
{
    orc_pixgeo g;
    if (scheme == 0) orc_ring_geo(nside, p, &g);
    else orc_nest_geo(nside, p, &g);
    *iring = g.iring;
    *jp = g.jp;
    return 0;
}

static int64_t orc_ring_from_geo(int64_t nside, int64_t iring, int64_t jp)
{
    const int64_t npix = 12 * nside * nside;
    const int64_t ncap = 2 * nside * (nside - 1);
    if (iring < nside) return 2 * iring * (iring - 1) + jp - 1;
    if (iring <= 3 * nside) return ncap + 4 * nside * (iring - nside) + jp - 1;
    int64_t i = 4 * nside - iring;
    return npix - 2 * i * (i + 1) + jp - 1;
}

/* NESTED -> RING index: through (ring, pixel-in-ring). */
int64_t orc_nest2ring(int nside, int64_t p)
{
    orc_pixgeo g;
    orc_nest_geo(nside, p, &g);
    return orc_ring_from_geo(nside, g.iring, g.jp);
}

/* (face, ix, iy) -> NESTED index */
static int64_t orc_xyf2nest(int64_t nside, int64_t ix, int64_t iy, int face)
{
    return (int64_t)face * nside * nside + orc_spread_bits(ix) + (orc_spread_bits(iy) << 1);
}

/* RING -> NESTED index: recover (face, ix, iy) from (ring, pixel-in-ring) by
 * inverting the NESTED geometry of orc_nest_geo over the 12 faces.  On the
 * right face ix+iy = jrll*N - ring - 1 and ix-iy = 2*jp - jpll*nr - 1 - kshift
 * (mod 8*nr); the admissible window |ix-iy| < N makes the face unique. */
int64_t orc_ring2nest(int nside, int64_t p)
{
    const int64_t N = nside;
    orc_pixgeo g;
    orc_ring_geo(N, p, &g);
    const int64_t mod = 8 * g.nr;
    for (int face = 0; face < 12; ++face) {
        int64_t s = (int64_t)orc_jrll[face] * N - g.iring - 1;
        if (s < 0 || s > 2 * N - 2) continue;
        int64_t d = 2 * g.jp - (int64_t)orc_jpll[face] * g.nr - 1 - g.kshift;
        d %= mod;
        if (d > mod / 2) d -= mod;
        if (d <= -mod / 2) d += mod;
        if (((s + d) & 1) != 0) continue;
        int64_t ix = (s + d) / 2, iy = (s - d) / 2;
        if (ix < 0 || iy < 0 || ix >= N || iy >= N) continue;
        return orc_xyf2nest(N, ix, iy, face);
    }
    return -1;
}

/* Ang -> pixel (HEALPix vec2pix), both schemes, long double. */
int64_t orc_vec2pix(int nside, int scheme, double x, double y, double zin)
{
    const long double N = nside;
    long double r = sqrtl((long double)x * x + (long double)y * y + (long double)zin * zin);
    long double z = zin / r;
    long double za = fabsl(z);
    long double phi = atan2l((long double)y, (long double)x);
    if (phi < 0) phi += 2.0L * ORC_PI_L;
    long double tt = phi / (0.5L * ORC_PI_L);   /* in [0,4) */
    if (tt >= 4.0L) tt -= 4.0L;
    int64_t ring;
    if (za <= 2.0L / 3.0L) {
        long double temp1 = N * (0.5L + tt);
        long double temp2 = N * z * 0.75L;
        int64_t jp = (int64_t)(temp1 - temp2);
        int64_t jm = (int64_t)(temp1 + temp2);
        int64_t ir = nside + 1 + jp - jm;           /* 1..2N+1 */
        int64_t kshift = 1 - (ir & 1);
        int64_t ip = (jp + jm - nside + kshift + 1) / 2;
        ip = ip % (4 * (int64_t)nside);
        ring = 2LL * nside * (nside - 1) + (ir - 1) * 4LL * nside + ip;
    } else {
        long double tp = tt - floorl(tt);
        long double tmp = N * sqrtl(3.0L * (1.0L - za));
        int64_t jp = (int64_t)(tp * tmp);
        int64_t jm = (int64_t)((1.0L - tp) * tmp);
        int64_t ir = jp + jm + 1;
        int64_t ip = (int64_t)(tt * ir);
        ip = ip % (4 * ir);
        if (z > 0) ring = 2 * ir * (ir - 1) + ip;
        else ring = 12LL * nside * nside - 2 * ir * (ir + 1) + ip;
    }
    return scheme == 0 ? ring : orc_ring2nest(nside, ring);
}

/* ------------------------------------------------------------------------ */
/* Sky direction convention (vissgen3d_blockage.cu:53-74)                    */
/* ------------------------------------------------------------------------ */

/* HEALPix unit vector (x, y, z) -> sky direction (l, m, n) of the reference:
 * lat = pi/2 - theta, phi' = -wrap(phi), l = cos(lat)cos(phi'),
 * m = cos(lat)sin(phi'), n = sin(lat)  ==  (x, -y, z).  Exact (a sign flip). */
void orc_lmn_from_xyz(int64_t n, const double *xyz, double *lmn)
{
    for (int64_t i = 0; i < n; ++i) {
        lmn[3 * i + 0] = xyz[3 * i + 0];
        lmn[3 * i + 1] = -xyz[3 * i + 1];
        lmn[3 * i + 2] = xyz[3 * i + 2];
    }
}

/* vissgen3d_blockage.cu:53-74 from FP32 theta/phi (the drop-in text inputs):
 * the angle edits are rounded to FP32 as the reference stores them, the trig
 * is FP64.  B is scaled by s (the pixel solid angle 4*pi/npix). */
void orc_sky_pre_f32(int64_t n, const float *theta, const float *phi, const float *B,
                     float s, double *lmn, float *Bout)
{
    for (int64_t i = 0; i < n; ++i) {
        float lat = (float)(M_PI / 2 - (double)theta[i]);
        float ph = phi[i];
        if ((double)ph > M_PI) ph = (float)((double)ph - 2 * M_PI);
        ph = -ph;
        double cl = cos((double)lat);
        lmn[3 * i + 0] = cl * cos((double)ph);
        lmn[3 * i + 1] = cl * sin((double)ph);
        lmn[3 * i + 2] = sin((double)lat);
        if (Bout) Bout[i] = B[i] * s;
    }
}

/* ------------------------------------------------------------------------ */
/* Occultation predicate (vissgen3d_blockage.cu:88-94,180-186,249-252)       */
/* ------------------------------------------------------------------------ */
/* An occulter is (q, thr): direction s is visible iff dot(s, q) >= thr, with
 * dot = fma(s2, q2, fma(s1, q1, s0*q0)) -- the same IEEE operations in the
 * CUDA kernels.  The reference's test acos(s.P/|P|) <= phi is this with
 * q = P/|P| and thr = cos(phi); the ray-sphere test against a Moon of radius
 * R is this with thr = -sqrt(1 - (R/|P|)^2); an Earth cap of radius rho
 * toward e is q = -e, thr = -cos(rho). */

static inline double orc_dot3(const double *s, const double *q)
{
    return fma(s[2], q[2], fma(s[1], q[1], s[0] * q[0]));
}

/* Reference cone threshold, vissgen3d_blockage.cu:249-252: the reference
 * computes theta = asinf(R/(R+h)) and phi = M_PI - theta on the host in FP32;
 * visible iff beta <= phi, i.e. dot >= cos(phi). */
double orc_cone_threshold(float R, float h)
{
    float th = asinf(R / (R + h));
    float ph = (float)(M_PI - (double)th);
    return cos((double)ph);
}

/* Occulter table from satellite positions P (n x 3, Moon-centred metres).
 * mode 0: ray-sphere against radius R (thr from |P|);
 * mode 1: fixed threshold fixed_thr (the reference cone).
 * occ is n x 4: (qx, qy, qz, thr). */
void orc_occulters(int64_t n, const double *P, double R, int mode, double fixed_thr,
                   double *occ)
{
    for (int64_t i = 0; i < n; ++i) {
        double x = P[3 * i], y = P[3 * i + 1], z = P[3 * i + 2];
        double r = sqrt(fma(z, z, fma(y, y, x * x)));
        occ[4 * i + 0] = x / r;
        occ[4 * i + 1] = y / r;
        occ[4 * i + 2] = z / r;
        if (mode == 0) {
            double rho = R / r;
            occ[4 * i + 3] = -sqrt(1.0 - rho * rho);
        } else {
            occ[4 * i + 3] = fixed_thr;
        }
    }
}

/* Visibility of (sample k, pixel j): AND over the sample's (up to 3) occulter
 * references; a negative reference is "no occulter". */
static inline int orc_visible(const int32_t *refs, const double *occ, const double *s)
{
    if (!refs) return 1;
    for (int c = 0; c < 3; ++c) {
        int32_t g = refs[c];
        if (g < 0) continue;
        const double *q = occ + 4 * (int64_t)g;
        if (!(orc_dot3(s, q) >= q[3])) return 0;
    }
    return 1;
}

/* The predicate's dot product, dot(s_i, q) in the exact operation order, for
 * building occulters whose threshold sits exactly on a pixel. */
void orc_dots(int64_t n, const double *lmn, const double *q4, double *out)
{
    for (int64_t i = 0; i < n; ++i) out[i] = orc_dot3(lmn + 3 * i, q4);
}

/* Mask bits: bit j of row k (rows of ceil(J/32) uint32 words). */
int orc_mask_bits(int64_t K, int64_t J, const double *lmn, const int32_t *refs,
                  const double *occ, uint32_t *bits)
{
    const int64_t W = (J + 31) / 32;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < K; ++k) {
        uint32_t *row = bits + k * W;
        memset(row, 0, sizeof(uint32_t) * W);
        for (int64_t j = 0; j < J; ++j)
            if (orc_visible(refs ? refs + 3 * k : NULL, occ, lmn + 3 * j))
                row[j >> 5] |= 1u << (j & 31);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Forward visibilities (vissgen3d_blockage.cu:76-102)                       */
/* ------------------------------------------------------------------------ */

/* Phase in turns of (sample k, pixel j): u.s + off, reduced to [-1/2, 1/2). */
static inline double orc_turns(const double *u, double off, const double *s)
{
    double t = fma(u[2], s[2], fma(u[1], s[1], u[0] * s[0])) + off;
    return t - nearbyint(t);
}

/* V_k = sum_j I_j vis_kj exp(-2 pi i (u_k.s_j + off_k)), k in [0,K).
 * uvw K x 3, off K (NULL = 0), lmn J x 3, I J, refs K x 3 (NULL = no mask),
 * V K x 2 (re, im).  The reference's w(n-1) convention (:95) is off_k = -w_k.
 * Accumulation in long double. */
int orc_forward(int64_t K, const double *uvw, const double *off, int64_t J,
                const double *lmn, const double *I, const int32_t *refs,
                const double *occ, double *V, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t k = 0; k < K; ++k) {
        long double re = 0, im = 0;
        const double *u = uvw + 3 * k;
        const double o = off ? off[k] : 0.0;
        const int32_t *rk = refs ? refs + 3 * k : NULL;
        for (int64_t j = 0; j < J; ++j) {
            const double *s = lmn + 3 * j;
            if (!orc_visible(rk, occ, s)) continue;
            double f = orc_turns(u, o, s);
            double sn, cs;
            sincos(2.0 * M_PI * f, &sn, &cs);
            re += (long double)I[j] * cs;
            im -= (long double)I[j] * sn;
        }
        V[2 * k] = (double)re;
        V[2 * k + 1] = (double)im;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Shell histogram and density compensation                                  */
/* (vissgen3d_blockage.cu:105-130, vissgen3d_noblockage.cu:132-141)          */
/* ------------------------------------------------------------------------ */

/* Shell index of a baseline length (in wavelengths), vissgen3d_blockage.cu:108:
 * ceil((bll - 1/4) / 0.5) in FP32 (the /0.5 is the exact *2). */
static inline int32_t orc_shell(float bll)
{
    volatile float d = bll - 0.25f;
    float c = ceilf(d * 2.0f);
    if (c != c) return -1;                       /* NaN: no shell */
    if (c > 1073741824.0f) return 1073741824;    /* saturate past 2^30 */
    if (c < -1073741824.0f) return -1073741824;
    return (int32_t)c;
}

/* gs[i] = shell index; counts[p-1] = multiplicity * #{i : gs[i] == p}, p in [1, nr]
 * (multiplicity 2 counts each unique row and its conjugate mirror);
 * dcf[0] = 1/(4 pi), dcf[k] = (2 pi / 3)(R^3 - (R - 1/2)^3) / counts[k-1]
 * with R = k/2 + 1/4 (the correct, un-shifted noblockage formula), FP64
 * rounded to FP32.  Any of gs/counts/dcf may be NULL. */
int orc_dcf(int64_t n, const float *bll, int nr, int multiplicity, int32_t *gs,
            uint32_t *counts, float *dcf)
{
    uint32_t *cnt = (uint32_t *)calloc((size_t)(nr > 0 ? nr : 1), sizeof(uint32_t));
    if (!cnt) return -1;
    for (int64_t i = 0; i < n; ++i) {
        int32_t g = orc_shell(bll[i]);
        if (gs) gs[i] = g;
        if (g >= 1 && g <= nr) cnt[g - 1]++;
    }
    for (int k = 0; k < nr; ++k) cnt[k] *= (uint32_t)multiplicity;
    if (counts) memcpy(counts, cnt, sizeof(uint32_t) * (size_t)nr);
    if (dcf) {
        dcf[0] = (float)(1.0 / (4.0 * M_PI));
        const double c = 2.0 * M_PI / 3.0;
        for (int k = 1; k <= nr; ++k) {
            double R = (double)k * 0.5 + 0.25;
            double Rm = R - 0.5;
            double vol = R * R * R - Rm * Rm * Rm;
            dcf[k] = (float)((c * vol) / (double)cnt[k - 1]);
        }
    }
    free(cnt);
    return 0;
}

/* Elevation factor dg (vissgen3d_blockage.cu:153-162):
 * gamma = asin(w/bll), dg = |sqrt(1 - 4 sin^2 gamma)| / |cos gamma| * 3/2,
 * evaluated without trig from x = w/bll: 1.5*sqrt(|1-4x^2|)/sqrt(1-x^2).
 * |x| >= 1 (and NaN) give +inf, which the 1/8 weight clamp then caps, as the
 * reference's fminf does with its NaN/inf. */
static inline float orc_dg(float w, float bll)
{
    double x = (double)w / (double)bll;
    if (!(fabs(x) < 1.0)) return INFINITY;
    double x2 = x * x;
    return (float)(1.5 * sqrt(fabs(1.0 - 4.0 * x2)) / sqrt(1.0 - x2));
}

int orc_gamma_dg(int64_t n, const float *w, const float *bll, float *dg)
{
    for (int64_t i = 0; i < n; ++i) dg[i] = orc_dg(w[i], bll[i]);
    return 0;
}

/* Per-row imaging weight, vissgen3d_blockage.cu:178,187:
 * min(dcf[gs] * dg, 1/8) in FP32; gs is clamped to [0, nr] (the reference
 * reads out of bounds there). */
int orc_weights(int64_t n, const int32_t *gs, const float *dg, const float *dcf, int nr,
                float *wt)
{
    for (int64_t i = 0; i < n; ++i) {
        int32_t g = gs[i] < 0 ? 0 : (gs[i] > nr ? nr : gs[i]);
        volatile float p = dcf[g] * dg[i];
        wt[i] = fminf(p, 0.125f);
    }
    return 0;
}

/* w-rotation V <- V exp(-2 pi i w) (vissgen3d_blockage.cu:150-151), FP64. */
int orc_wrot(int64_t n, const double *w, double *V)
{
    for (int64_t i = 0; i < n; ++i) {
        double f = w[i] - nearbyint(w[i]);
        double sn, cs;
        sincos(2.0 * M_PI * f, &sn, &cs);
        double re = V[2 * i], im = V[2 * i + 1];
        V[2 * i] = re * cs + im * sn;
        V[2 * i + 1] = im * cs - re * sn;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Imaging adjoint (vissgen3d_blockage.cu:167-192)                            */
/* ------------------------------------------------------------------------ */

/* C_j = sum_k Re(a_k exp(+2 pi i (u_k.s_j + off_k))) vis_kj, j in [0,J).
 * a is K x 2 (the weighted visibilities w_k V_k).  refs NULL = no mask (the
 * noblockage imaging, vissgen3d_noblockage.cu:167-182).  Long double sums. */
int orc_adjoint(int64_t K, const double *uvw, const double *off, const double *a,
                int64_t J, const double *lmn, const int32_t *refs, const double *occ,
                double *C, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t j = 0; j < J; ++j) {
        long double acc = 0;
        const double *s = lmn + 3 * j;
        for (int64_t k = 0; k < K; ++k) {
            if (!orc_visible(refs ? refs + 3 * k : NULL, occ, s)) continue;
            double f = orc_turns(uvw + 3 * k, off ? off[k] : 0.0, s);
            double sn, cs;
            sincos(2.0 * M_PI * f, &sn, &cs);
            acc += (long double)a[2 * k] * cs - (long double)a[2 * k + 1] * sn;
        }
        C[j] = (double)acc;
    }
    return 0;
}

/* Phase-derivative sums used by the position gradient:
 * D_k = sum_j I_j vis_kj s_j exp(-2 pi i (u_k.s_j + off_k)),  D is K x 3 x 2. */
int orc_forward_dphase(int64_t K, const double *uvw, const double *off, int64_t J,
                       const double *lmn, const double *I, const int32_t *refs,
                       const double *occ, double *D, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t k = 0; k < K; ++k) {
        long double acc[6] = {0, 0, 0, 0, 0, 0};
        const double *u = uvw + 3 * k;
        const double o = off ? off[k] : 0.0;
        const int32_t *rk = refs ? refs + 3 * k : NULL;
        for (int64_t j = 0; j < J; ++j) {
            const double *s = lmn + 3 * j;
            if (!orc_visible(rk, occ, s)) continue;
            double f = orc_turns(u, o, s);
            double sn, cs;
            sincos(2.0 * M_PI * f, &sn, &cs);
            for (int c = 0; c < 3; ++c) {
                acc[2 * c] += (long double)I[j] * s[c] * cs;
                acc[2 * c + 1] -= (long double)I[j] * s[c] * sn;
            }
        }
        for (int c = 0; c < 6; ++c) D[6 * k + c] = (double)acc[c];
    }
    return 0;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
