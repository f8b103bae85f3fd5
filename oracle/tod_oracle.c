/*
 * tod_oracle.c -- CPU restatement of the reference beam-convolution TOD path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of the benchmark load it.  Nothing in
 * the product package links or calls it.
 *
 * What it restates (file:line in ArtemBasyrov/tod_generation_mapbased_beam):
 *   numba_healpy.py:53-70    ring_above          -> orc_ring_above
 *   numba_healpy.py:73-101   ring_info           -> orc_ring_info
 *   numba_healpy.py:104-114  ring_z              -> orc_ring_z
 *   numba_healpy.py:120-236  get_interp_weights  -> oracle_get_interp_weights
 *   numba_healpy.py:358-499  ring interp + angles-> orc_ring_interp
 *   numba_healpy.py:505-535  pix2ang (RING)      -> oracle_pix2ang
 *   numba_healpy.py:642-693  ang2pix (RING)      -> oracle_ang2pix
 *   tod_rotations.py:83-134  double Rodrigues    -> orc_rodrigues
 *   tod_bilinear.py:84-145   spin-2 cos2d/sin2d  -> orc_spin2
 *   tod_bilinear.py:151-199  per-sample cache    -> orc_spin2_cached
 *   tod_bilinear.py:205-477  fused bilinear      -> oracle_gather_accum_bilinear
 *   tod_nearest.py:21-158    fused nearest       -> oracle_gather_accum_nearest
 *
 * Arithmetic follows the reference operation by operation (left-to-right
 * evaluation, no FMA contraction: build with -ffp-contract=off), Python float
 * modulo semantics for `%`, and x86 truncation semantics for int() (NaN or
 * out-of-range -> INT64_MIN, as cvttsd2si does).  Transcendentals come from
 * the host libm, as the Numba kernels' do.
 *
 * Operand types follow the reference kernels: they read every float32 input
 * with float(arr[i]), which Numba types as float32, so the recentring
 * Rodrigues step mixes float32 and float64 arithmetic and the boresight
 * longitude comes from the C library's atan2f.  With params_f64 = 1 the same
 * entry points take float64 parameters and compute everything in float64:
 * that is the FP64 "ideal" oracle used for the error budget of the reduced-
 * precision forms.
 *
 * Map reads are bounds-checked: an index outside [0, npix) (possible only for
 * NaN pointing, or for the spill into ring 4*nside of the reference's phi
 * modulo) contributes nothing and is counted in the returned error count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_TWO_PI (2.0 * 3.141592653589793)
#define ORC_PI 3.141592653589793
#define ORC_TWO_THIRDS (2.0 / 3.0)
#define ORC_CACHE_SIZE 1024
#define ORC_CACHE_MASK (ORC_CACHE_SIZE - 1)
#define ORC_CACHE_HASH 2654435769LL

/* int() of a float64 with x86 cvttsd2si semantics. */
static inline int64_t orc_int(double x) {
    if (!(x >= -9223372036854775808.0 && x < 9223372036854775808.0))
        return INT64_MIN;
    return (int64_t)x;
}

/* Wrapping int64 arithmetic (Numba integers wrap on overflow). */
static inline int64_t orc_add(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
static inline int64_t orc_sub(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }

/* Python `a % n` for integers with n > 0 (result in [0, n)). */
static inline int64_t orc_imod(int64_t a, int64_t n) {
    int64_t r = a % n;
    return r < 0 ? r + n : r;
}

/* Python `x % w` for floats (CPython float_rem / Numba real_divmod). */
static inline double orc_fmod(double x, double w) {
    double m = fmod(x, w);
    if (m != 0.0) {
        if ((w < 0.0) != (m < 0.0)) m += w;
    } else {
        m = (w < 0.0) ? -0.0 : 0.0;
    }
    return m;
}

static inline double orc_max0(double x) { return x > 0.0 ? x : 0.0; }
static inline double orc_clamp1(double x) {
    double a = (x < 1.0) ? x : 1.0;   /* min(1.0, x) */
    return (a > -1.0) ? a : -1.0;     /* max(-1.0, .) */
}

static int64_t orc_ring_above(int64_t nside, double z) {
    double az = fabs(z);
    int64_t ir;
    if (az > ORC_TWO_THIRDS) {
        double tp = (double)nside * sqrt(3.0 * (1.0 - az));
        ir = orc_int(tp);
        if (z < 0.0) ir = orc_sub(orc_sub(4 * nside, ir), 1);
    } else {
        ir = orc_int((double)nside * (2.0 - 1.5 * z));
    }
    return ir;
}

static void orc_ring_info(int64_t nside, int64_t ir, int64_t npix, int64_t *n_pix,
                          int64_t *first_pix, double *phi0, double *dphi) {
    int64_t n, fp, s;
    if (ir < nside) {
        n = 4 * ir;
        fp = 2 * ir * (ir - 1);
        s = 1;
    } else if (ir <= 3 * nside) {
        n = 4 * nside;
        fp = 2 * nside * (nside - 1) + (ir - nside) * 4 * nside;
        s = (orc_imod(ir - nside, 2) == 0) ? 1 : 0;
    } else {
        int64_t i2 = 4 * nside - ir;
        n = 4 * i2;
        fp = npix - 2 * i2 * (i2 + 1);
        s = 1;
    }
    double dp = ORC_TWO_PI / (double)n;
    *n_pix = n;
    *first_pix = fp;
    *dphi = dp;
    *phi0 = (double)s * dp * 0.5;
}

static double orc_ring_z(int64_t nside, int64_t ir) {
    if (ir < nside) {
        double t = (double)ir;
        return 1.0 - t * t / (3.0 * (double)nside * (double)nside);
    } else if (ir <= 3 * nside) {
        return ORC_TWO_THIRDS * (2.0 - (double)ir / (double)nside);
    } else {
        double t = (double)(4 * nside - ir);
        return -(1.0 - t * t / (3.0 * (double)nside * (double)nside));
    }
}

/* 4-neighbour RING stencil with neighbour (z, phi) (numba_healpy.py:358-499). */
typedef struct {
    int64_t p[4];
    double w[4];
    double zn[4];
    double phin[4];
} orc_stencil;

static void orc_ring_interp(int64_t nside, double z, double phi_w, int64_t npix, orc_stencil *st) {
    int64_t ir_above = orc_ring_above(nside, z);
    int64_t ir_below = orc_add(ir_above, 1);
    if (ir_above == 0) {
        int64_t na, fpa;
        double phi0a, dphia;
        orc_ring_info(nside, 1, npix, &na, &fpa, &phi0a, &dphia);
        double tw = orc_fmod((phi_w - phi0a) / dphia, (double)na);
        int64_t ip = orc_int(tw);
        double frac = tw - (double)ip;
        int64_t ip2 = orc_imod(orc_add(ip, 1), na);
        int64_t o1 = orc_imod(orc_add(ip, 2), na), o2 = orc_imod(ip2 + 2, na);
        st->p[0] = fpa + o1;
        st->p[1] = fpa + o2;
        st->p[2] = orc_add(fpa, ip);
        st->p[3] = fpa + ip2;
        double za = orc_ring_z(nside, 1);
        double ta = acos(za);
        double theta = acos(z);
        double wt = theta / ta;
        double nf = (1.0 - wt) * 0.25;
        st->w[0] = nf;
        st->w[1] = nf;
        st->w[2] = (1.0 - frac) * wt + nf;
        st->w[3] = frac * wt + nf;
        for (int k = 0; k < 4; ++k) st->zn[k] = za;
        st->phin[0] = phi0a + (double)o1 * dphia;
        st->phin[1] = phi0a + (double)o2 * dphia;
        st->phin[2] = phi0a + (double)ip * dphia;
        st->phin[3] = phi0a + (double)ip2 * dphia;
    } else if (ir_below == 4 * nside) {
        int64_t ir_last = 4 * nside - 1;
        int64_t na, fpa;
        double phi0a, dphia;
        orc_ring_info(nside, ir_last, npix, &na, &fpa, &phi0a, &dphia);
        double tw = orc_fmod((phi_w - phi0a) / dphia, (double)na);
        int64_t ip = orc_int(tw);
        double frac = tw - (double)ip;
        int64_t ip2 = orc_imod(orc_add(ip, 1), na);
        int64_t o1 = orc_imod(orc_add(ip, 2), na), o2 = orc_imod(ip2 + 2, na);
        st->p[0] = orc_add(fpa, ip);
        st->p[1] = fpa + ip2;
        st->p[2] = fpa + o1;
        st->p[3] = fpa + o2;
        double za = orc_ring_z(nside, ir_last);
        double ta = acos(za);
        double theta = acos(z);
        double ws = (theta - ta) / (ORC_PI - ta);
        double sf = ws * 0.25;
        st->w[0] = (1.0 - frac) * (1.0 - ws) + sf;
        st->w[1] = frac * (1.0 - ws) + sf;
        st->w[2] = sf;
        st->w[3] = sf;
        for (int k = 0; k < 4; ++k) st->zn[k] = za;
        st->phin[0] = phi0a + (double)ip * dphia;
        st->phin[1] = phi0a + (double)ip2 * dphia;
        st->phin[2] = phi0a + (double)o1 * dphia;
        st->phin[3] = phi0a + (double)o2 * dphia;
    } else {
        double za = orc_ring_z(nside, ir_above);
        double zb = orc_ring_z(nside, ir_below);
        double ta = acos(za);
        double tb = acos(zb);
        double theta = acos(z);
        double wb = (theta - ta) / (tb - ta);
        double wa = 1.0 - wb;
        int64_t na, fpa, nb, fpb;
        double phi0a, dphia, phi0b, dphib;
        orc_ring_info(nside, ir_above, npix, &na, &fpa, &phi0a, &dphia);
        double tw = orc_fmod((phi_w - phi0a) / dphia, (double)na);
        int64_t ia = orc_int(tw);
        double fa = tw - (double)ia;
        int64_t ia1 = orc_imod(orc_add(ia, 1), na);
        st->p[0] = orc_add(fpa, ia);
        st->p[1] = fpa + ia1;
        st->w[0] = wa * (1.0 - fa);
        st->w[1] = wa * fa;
        orc_ring_info(nside, ir_below, npix, &nb, &fpb, &phi0b, &dphib);
        tw = orc_fmod((phi_w - phi0b) / dphib, (double)nb);
        int64_t ib = orc_int(tw);
        double fb = tw - (double)ib;
        int64_t ib1 = orc_imod(orc_add(ib, 1), nb);
        st->p[2] = orc_add(fpb, ib);
        st->p[3] = fpb + ib1;
        st->w[2] = wb * (1.0 - fb);
        st->w[3] = wb * fb;
        st->zn[0] = za;
        st->zn[1] = za;
        st->zn[2] = zb;
        st->zn[3] = zb;
        st->phin[0] = phi0a + (double)ia * dphia;
        st->phin[1] = phi0a + (double)ia1 * dphia;
        st->phin[2] = phi0b + (double)ib * dphib;
        st->phin[3] = phi0b + (double)ib1 * dphib;
    }
}

/* Double Rodrigues: recentre about k, then roll about the boresight p
 * (tod_rotations.py:83-134), all float64 (the "ideal" oracle). */
static inline void orc_rodrigues(double vx, double vy, double vz, double kx, double ky,
                                 double kz, double ca, double sa, double px, double py,
                                 double pz, double cp, double sp, double *ox, double *oy,
                                 double *oz) {
    double oma = 1.0 - ca;
    double omp = 1.0 - cp;
    double dkv = kx * vx + ky * vy + kz * vz;
    double rx = vx * ca + (ky * vz - kz * vy) * sa + kx * dkv * oma;
    double ry = vy * ca + (kz * vx - kx * vz) * sa + ky * dkv * oma;
    double rz = vz * ca + (kx * vy - ky * vx) * sa + kz * dkv * oma;
    double dpr = px * rx + py * ry + pz * rz;
    *ox = rx * cp + (py * rz - pz * ry) * sp + px * dpr * omp;
    *oy = ry * cp + (pz * rx - px * rz) * sp + py * dpr * omp;
    *oz = rz * cp + (px * ry - py * rx) * sp + pz * dpr * omp;
}

/* The same rotation with the reference kernels' operand types.  The kernels
 * load every parameter with float(arr[i]), which Numba types as float32 for
 * float32 arrays, so the recentre step mixes float32 products/sums with the
 * float64 (1 - cos) factor; the roll step is float64 with widened inputs
 * (tod_bilinear.py:294-328 calling tod_rotations.py:122-133). */
static inline void orc_rodrigues_ref32(float vx, float vy, float vz, float kx, float ky,
                                       float kz, float ca, float sa, float px, float py,
                                       float pz, float cp, float sp, double *ox, double *oy,
                                       double *oz) {
    double oma = 1.0 - (double)ca;
    double omp = 1.0 - (double)cp;
    float dkv = kx * vx + ky * vy + kz * vz;
    float ax = vx * ca + (ky * vz - kz * vy) * sa;
    float ay = vy * ca + (kz * vx - kx * vz) * sa;
    float az = vz * ca + (kx * vy - ky * vx) * sa;
    double rx = (double)ax + (double)(kx * dkv) * oma;
    double ry = (double)ay + (double)(ky * dkv) * oma;
    double rz = (double)az + (double)(kz * dkv) * oma;
    double dpx = px, dpy = py, dpz = pz, dcp = cp, dsp = sp;
    double dpr = dpx * rx + dpy * ry + dpz * rz;
    *ox = rx * dcp + (dpy * rz - dpz * ry) * dsp + dpx * dpr * omp;
    *oy = ry * dcp + (dpz * rx - dpx * rz) * dsp + dpy * dpr * omp;
    *oz = rz * dcp + (dpx * ry - dpy * rx) * dsp + dpz * dpr * omp;
}

/* Per-sample parameters in either precision. */
typedef struct {
    const void *vec, *axes, *ca, *sa, *pts, *cp, *sp;
    int f64;
} orc_params;

static inline void orc_rotate(const orc_params *P, int64_t b, int64_t s, double *ox, double *oy,
                              double *oz) {
    if (P->f64) {
        const double *v = (const double *)P->vec + 3 * s, *k = (const double *)P->axes + 3 * b;
        const double *p = (const double *)P->pts + 3 * b;
        orc_rodrigues(v[0], v[1], v[2], k[0], k[1], k[2], ((const double *)P->ca)[b],
                      ((const double *)P->sa)[b], p[0], p[1], p[2], ((const double *)P->cp)[b],
                      ((const double *)P->sp)[b], ox, oy, oz);
    } else {
        const float *v = (const float *)P->vec + 3 * s, *k = (const float *)P->axes + 3 * b;
        const float *p = (const float *)P->pts + 3 * b;
        orc_rodrigues_ref32(v[0], v[1], v[2], k[0], k[1], k[2], ((const float *)P->ca)[b],
                            ((const float *)P->sa)[b], p[0], p[1], p[2],
                            ((const float *)P->cp)[b], ((const float *)P->sp)[b], ox, oy, oz);
    }
}

/* Boresight (z, sin theta, phi) used by the spin-2 angle.  Reference typing:
 * z = clamp(float64(bz)); sin = sqrt(1 - float32(bz*bz)); phi = atan2f(by, bx)
 * widened, + 2pi if negative (tod_bilinear.py:306-310, tod_nearest.py:85-89). */
static inline void orc_boresight(const orc_params *P, int64_t b, double *z, double *sth,
                                 double *phi) {
    if (P->f64) {
        const double *p = (const double *)P->pts + 3 * b;
        *z = orc_clamp1(p[2]);
        *sth = sqrt(orc_max0(1.0 - p[2] * p[2]));
        *phi = atan2(p[1], p[0]);
    } else {
        const float *p = (const float *)P->pts + 3 * b;
        float bz2 = p[2] * p[2];
        *z = orc_clamp1((double)p[2]);
        *sth = sqrt(orc_max0(1.0 - (double)bz2));
        *phi = (double)atan2f(p[1], p[0]);
    }
    if (*phi < 0.0) *phi += ORC_TWO_PI;
}

/* cos 2d, sin 2d of the pixel -> boresight frame rotation (tod_bilinear.py:84-145). */
static inline void orc_spin2(double z_pix, double sth_pix, double phi_pix, double z_pts,
                             double sth_pts, double phi_pts, double *c2d, double *s2d) {
    if (phi_pts == phi_pix && sth_pts == sth_pix && z_pts == z_pix) {
        *c2d = 1.0;
        *s2d = 0.0;
        return;
    }
    double dphi = phi_pts - phi_pix;
    double ch = cos(dphi * 0.5);
    double sh = sin(dphi * 0.5);
    double sin_dphi = 2.0 * ch * sh;
    double cos_dphi = 1.0 - 2.0 * sh * sh;
    double sh2 = sh * sh;
    double dz = z_pts - z_pix;
    double ds = sth_pts - sth_pix;
    double st2 = 0.25 * (dz * dz + ds * ds);
    double S = sth_pix * sth_pts;
    double h = st2 + S * sh2;
    double sin2_dtheta = 4.0 * st2 * (1.0 - st2);
    double z_sum = z_pts + z_pix;
    double N = 2.0 * sin_dphi * z_sum * h;
    double C = z_pts * z_pix;
    double term1 = sin2_dtheta * cos_dphi;
    double term2 = 4.0 * S * C * sh2 * sh2;
    double term3 = S * sin_dphi * sin_dphi;
    double D = term1 - term2 + term3;
    double u = 1.0 / (N * N + D * D);
    *c2d = (D * D - N * N) * u;
    *s2d = 2.0 * N * D * u;
}

typedef struct {
    int64_t pix[ORC_CACHE_SIZE];
    double c2d[ORC_CACHE_SIZE];
    double s2d[ORC_CACHE_SIZE];
} orc_cache;

/* Direct-mapped per-sample spin-2 cache (tod_bilinear.py:151-199). */
static inline void orc_spin2_cached(int64_t p, double z_n, double phi_n, double z_pts,
                                    double sth_pts, double phi_pts, orc_cache *cc,
                                    double *c2d, double *s2d) {
    int64_t slot = (int64_t)(((uint64_t)p * (uint64_t)ORC_CACHE_HASH) & ORC_CACHE_MASK);
    if (cc->pix[slot] == p) {
        *c2d = cc->c2d[slot];
        *s2d = cc->s2d[slot];
        return;
    }
    double sth_n = sqrt(orc_max0(1.0 - z_n * z_n));
    orc_spin2(z_n, sth_n, phi_n, z_pts, sth_pts, phi_pts, c2d, s2d);
    cc->pix[slot] = p;
    cc->c2d[slot] = *c2d;
    cc->s2d[slot] = *s2d;
}

static inline double orc_map(const void *mp, int map_f64, int64_t stride, int64_t c, int64_t p) {
    if (map_f64) return ((const double *)mp)[c * stride + p];
    return (double)((const float *)mp)[c * stride + p];
}

/* mp[c, p] * bv as the nearest kernel types it (tod_nearest.py:146, :158): the
 * map element is not passed through float(), so a float32 map times the
 * float32 beam weight is a float32 product, widened when added to tod. */
static inline double orc_map_x_beam(const void *mp, int map_f64, int64_t stride, int64_t c,
                                    int64_t p, double bv) {
    if (map_f64) return ((const double *)mp)[c * stride + p] * bv;
    return (double)(((const float *)mp)[c * stride + p] * (float)bv);
}

static void orc_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* Fused bilinear kernel (tod_bilinear.py:205-477).
 *   vec (S,3) and the six per-sample parameter arrays: float32 with the
 *   reference's operand typing (params_f64 == 0) or float64 (ideal oracle);
 *   beam (S,) float64 (the float32 weights widened exactly);
 *   map (C, stride) float32 or float64; tod (C,B) float64 accumulated in place.
 * Returns the number of skipped out-of-range map reads. */
int64_t oracle_gather_accum_bilinear(const void *vec, const void *axes, const void *ca_,
                                     const void *sa_, const void *pts, const void *cp_,
                                     const void *sp_, int params_f64, int64_t nside,
                                     const void *mp, int map_f64, int64_t C, int64_t map_stride,
                                     const double *beam, int64_t B, int64_t S, double *tod,
                                     int64_t c_q, int64_t c_u, int nthreads) {
    const int64_t npix = 12 * nside * nside;
    const int has_qu = (c_q >= 0 && c_u >= 0);
    const orc_params P = {vec, axes, ca_, sa_, pts, cp_, sp_, params_f64};
    int64_t other[16];
    int64_t n_other = 0;
    for (int64_t c = 0; c < C && n_other < 16; ++c)
        if (c != c_q && c != c_u) other[n_other++] = c;
    int64_t errors = 0;
    orc_set_threads(nthreads);
#pragma omp parallel reduction(+ : errors)
    {
        orc_cache *cc = has_qu ? (orc_cache *)malloc(sizeof(orc_cache)) : NULL;
#pragma omp for schedule(dynamic, 64)
        for (int64_t b = 0; b < B; ++b) {
            double z_pts = 0.0, sth_pts = 0.0, phi_pts = 0.0;
            if (has_qu) {
                for (int i = 0; i < ORC_CACHE_SIZE; ++i) cc->pix[i] = -1;
                orc_boresight(&P, b, &z_pts, &sth_pts, &phi_pts);
            }
            for (int64_t s = 0; s < S; ++s) {
                double vx, vy, vz;
                orc_rotate(&P, b, s, &vx, &vy, &vz);
                double z = orc_clamp1(vz);
                double phi_w = atan2(vy, vx);
                if (phi_w < 0.0) phi_w += ORC_TWO_PI;
                double bv = beam[s];
                orc_stencil st;
                orc_ring_interp(nside, z, phi_w, npix, &st);
                int ok = 1;
                for (int k = 0; k < 4; ++k)
                    if (st.p[k] < 0 || st.p[k] >= npix) ok = 0;
                if (!ok) {
                    errors += 1;
                    continue;
                }
                if (has_qu) {
                    double c2[4], s2[4];
                    for (int k = 0; k < 4; ++k)
                        orc_spin2_cached(st.p[k], st.zn[k], st.phin[k], z_pts, sth_pts, phi_pts,
                                         cc, &c2[k], &s2[k]);
                    double q[4], u[4];
                    for (int k = 0; k < 4; ++k) {
                        q[k] = orc_map(mp, map_f64, map_stride, c_q, st.p[k]);
                        u[k] = orc_map(mp, map_f64, map_stride, c_u, st.p[k]);
                    }
                    tod[c_q * B + b] += (st.w[0] * (q[0] * c2[0] + u[0] * s2[0]) +
                                         st.w[1] * (q[1] * c2[1] + u[1] * s2[1]) +
                                         st.w[2] * (q[2] * c2[2] + u[2] * s2[2]) +
                                         st.w[3] * (q[3] * c2[3] + u[3] * s2[3])) * bv;
                    tod[c_u * B + b] += (st.w[0] * (-q[0] * s2[0] + u[0] * c2[0]) +
                                         st.w[1] * (-q[1] * s2[1] + u[1] * c2[1]) +
                                         st.w[2] * (-q[2] * s2[2] + u[2] * c2[2]) +
                                         st.w[3] * (-q[3] * s2[3] + u[3] * c2[3])) * bv;
                    for (int64_t oi = 0; oi < n_other; ++oi) {
                        int64_t c = other[oi];
                        tod[c * B + b] += (st.w[0] * orc_map(mp, map_f64, map_stride, c, st.p[0]) +
                                           st.w[1] * orc_map(mp, map_f64, map_stride, c, st.p[1]) +
                                           st.w[2] * orc_map(mp, map_f64, map_stride, c, st.p[2]) +
                                           st.w[3] * orc_map(mp, map_f64, map_stride, c, st.p[3])) * bv;
                    }
                } else {
                    for (int64_t c = 0; c < C; ++c) {
                        tod[c * B + b] += (st.w[0] * orc_map(mp, map_f64, map_stride, c, st.p[0]) +
                                           st.w[1] * orc_map(mp, map_f64, map_stride, c, st.p[1]) +
                                           st.w[2] * orc_map(mp, map_f64, map_stride, c, st.p[2]) +
                                           st.w[3] * orc_map(mp, map_f64, map_stride, c, st.p[3])) * bv;
                    }
                }
            }
        }
        free(cc);
    }
    return errors;
}

/* Fused nearest-pixel kernel (tod_nearest.py:21-158). Same argument meaning. */
int64_t oracle_gather_accum_nearest(const void *vec, const void *axes, const void *ca_,
                                    const void *sa_, const void *pts, const void *cp_,
                                    const void *sp_, int params_f64, int64_t nside,
                                    const void *mp, int map_f64, int64_t C, int64_t map_stride,
                                    const double *beam, int64_t B, int64_t S, double *tod,
                                    int64_t c_q, int64_t c_u, int nthreads) {
    const int64_t npix = 12 * nside * nside;
    const int has_qu = (c_q >= 0 && c_u >= 0);
    const orc_params P = {vec, axes, ca_, sa_, pts, cp_, sp_, params_f64};
    int64_t errors = 0;
    orc_set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : errors)
    for (int64_t b = 0; b < B; ++b) {
        double bz_pts, bsth_pts, bphi_pts;
        orc_boresight(&P, b, &bz_pts, &bsth_pts, &bphi_pts);
        for (int64_t s = 0; s < S; ++s) {
            double vx, vy, vz;
            orc_rotate(&P, b, s, &vx, &vy, &vz);
            double phi_w = atan2(vy, vx);
            if (phi_w < 0.0) phi_w += ORC_TWO_PI;
            double z = vz;
            double sin_th = sqrt(orc_max0(vx * vx + vy * vy));
            int64_t ir_above = orc_ring_above(nside, z);
            if (ir_above < 1)
                ir_above = 1;
            else if (ir_above > 4 * nside - 2)
                ir_above = 4 * nside - 2;
            int64_t best_pix = 0;
            double best_cos = -2.0, best_zc = 0.0, best_phic = 0.0;
            for (int g = 0; g < 2; ++g) {
                int64_t ir = ir_above + g;
                if (ir < 1 || ir > 4 * nside - 1) continue;
                int64_t n, fp;
                double phi0, dphi;
                orc_ring_info(nside, ir, npix, &n, &fp, &phi0, &dphi);
                double zc = orc_ring_z(nside, ir);
                double szc = sqrt(orc_max0(1.0 - zc * zc));
                int64_t ipb = orc_imod(orc_int(phi_w * (double)n / ORC_TWO_PI), n);
                for (int t = 0; t < 2; ++t) {
                    int64_t ip = t == 0 ? ipb : orc_imod(ipb + 1, n);
                    double phic = phi0 + (double)ip * dphi;
                    double cosd = sin_th * szc * cos(phi_w - phic) + z * zc;
                    if (cosd > best_cos) {
                        best_cos = cosd;
                        best_pix = fp + ip;
                        best_zc = zc;
                        best_phic = phic;
                    }
                }
            }
            if (best_pix < 0 || best_pix >= npix) {
                errors += 1;
                continue;
            }
            double bv = beam[s];
            if (!has_qu) {
                for (int64_t c = 0; c < C; ++c)
                    tod[c * B + b] += orc_map_x_beam(mp, map_f64, map_stride, c, best_pix, bv);
            } else {
                double sth_n = sqrt(orc_max0(1.0 - best_zc * best_zc));
                double c2d, s2d;
                orc_spin2(best_zc, sth_n, best_phic, bz_pts, bsth_pts, bphi_pts, &c2d, &s2d);
                double qv = orc_map(mp, map_f64, map_stride, c_q, best_pix);
                double uv = orc_map(mp, map_f64, map_stride, c_u, best_pix);
                tod[c_q * B + b] += (qv * c2d + uv * s2d) * bv;
                tod[c_u * B + b] += (-qv * s2d + uv * c2d) * bv;
                for (int64_t c = 0; c < C; ++c)
                    if (c != c_q && c != c_u)
                        tod[c * B + b] += orc_map_x_beam(mp, map_f64, map_stride, c, best_pix, bv);
            }
        }
    }
    return errors;
}

/* Per-(b,s) stencil of the fused bilinear path, for pixel-level comparisons:
 * pix (4, B*S) int64, wgt (4, B*S) float64, n = b*S + s. */
void oracle_bilinear_stencils(const void *vec, const void *axes, const void *ca_,
                              const void *sa_, const void *pts, const void *cp_,
                              const void *sp_, int params_f64, int64_t nside, int64_t B,
                              int64_t S, int64_t *pix, double *wgt, int nthreads) {
    const int64_t npix = 12 * nside * nside;
    const int64_t BS = B * S;
    const orc_params P = {vec, axes, ca_, sa_, pts, cp_, sp_, params_f64};
    orc_set_threads(nthreads);
#pragma omp parallel for schedule(static)
    for (int64_t b = 0; b < B; ++b) {
        for (int64_t s = 0; s < S; ++s) {
            double vx, vy, vz;
            orc_rotate(&P, b, s, &vx, &vy, &vz);
            double z = orc_clamp1(vz);
            double phi_w = atan2(vy, vx);
            if (phi_w < 0.0) phi_w += ORC_TWO_PI;
            orc_stencil st;
            orc_ring_interp(nside, z, phi_w, npix, &st);
            int64_t n = b * S + s;
            for (int k = 0; k < 4; ++k) {
                pix[k * BS + n] = st.p[k];
                wgt[k * BS + n] = st.w[k];
            }
        }
    }
}

/* atan2f of the host C library, as the reference's float32 math.atan2 uses. */
void oracle_atan2f(const float *y, const float *x, int64_t N, float *out) {
    for (int64_t i = 0; i < N; ++i) out[i] = atan2f(y[i], x[i]);
}

/* hp.get_interp_weights restatement (numba_healpy.py:120-236): theta-based. */
void oracle_get_interp_weights(int64_t nside, const double *theta, const double *phi, int64_t N,
                               int64_t *pix, double *wgt) {
    const int64_t npix = 12 * nside * nside;
    for (int64_t i = 0; i < N; ++i) {
        double th = theta[i], ph = phi[i];
        double z = cos(th);
        int64_t ir_above = orc_ring_above(nside, z);
        int64_t ir_below = orc_add(ir_above, 1);
        int64_t p[4];
        double w[4];
        if (ir_above == 0) {
            int64_t na, fpa;
            double phi0a, dphia;
            orc_ring_info(nside, 1, npix, &na, &fpa, &phi0a, &dphia);
            double tw = orc_fmod((ph - phi0a) / dphia, (double)na);
            int64_t ip = orc_int(tw);
            double frac = tw - (double)ip;
            int64_t ip2 = orc_imod(orc_add(ip, 1), na);
            p[2] = orc_add(fpa, ip);
            p[3] = fpa + ip2;
            p[0] = orc_imod(orc_add(ip, 2), na);
            p[1] = orc_imod(ip2 + 2, na);
            double ta = acos(orc_ring_z(nside, 1));
            double wt = th / ta;
            double nf = (1.0 - wt) * 0.25;
            w[0] = nf;
            w[1] = nf;
            w[2] = (1.0 - frac) * wt + nf;
            w[3] = frac * wt + nf;
        } else if (ir_below == 4 * nside) {
            int64_t ir_last = 4 * nside - 1;
            int64_t na, fpa;
            double phi0a, dphia;
            orc_ring_info(nside, ir_last, npix, &na, &fpa, &phi0a, &dphia);
            double tw = orc_fmod((ph - phi0a) / dphia, (double)na);
            int64_t ip = orc_int(tw);
            double frac = tw - (double)ip;
            int64_t ip2 = orc_imod(orc_add(ip, 1), na);
            p[0] = orc_add(fpa, ip);
            p[1] = fpa + ip2;
            p[2] = orc_imod(orc_add(ip, 2), na) + fpa;
            p[3] = orc_imod(ip2 + 2, na) + fpa;
            double ta = acos(orc_ring_z(nside, ir_last));
            double ws = (th - ta) / (ORC_PI - ta);
            double sf = ws * 0.25;
            w[0] = (1.0 - frac) * (1.0 - ws) + sf;
            w[1] = frac * (1.0 - ws) + sf;
            w[2] = sf;
            w[3] = sf;
        } else {
            double ta = acos(orc_ring_z(nside, ir_above));
            double tb = acos(orc_ring_z(nside, ir_below));
            double wb = (th - ta) / (tb - ta);
            double wa = 1.0 - wb;
            int64_t na, fpa, nb, fpb;
            double phi0a, dphia, phi0b, dphib;
            orc_ring_info(nside, ir_above, npix, &na, &fpa, &phi0a, &dphia);
            double tw = orc_fmod((ph - phi0a) / dphia, (double)na);
            int64_t ia = orc_int(tw);
            double fa = tw - (double)ia;
            p[0] = orc_add(fpa, ia);
            p[1] = fpa + orc_imod(orc_add(ia, 1), na);
            w[0] = wa * (1.0 - fa);
            w[1] = wa * fa;
            orc_ring_info(nside, ir_below, npix, &nb, &fpb, &phi0b, &dphib);
            tw = orc_fmod((ph - phi0b) / dphib, (double)nb);
            int64_t ib = orc_int(tw);
            double fb = tw - (double)ib;
            p[2] = orc_add(fpb, ib);
            p[3] = fpb + orc_imod(orc_add(ib, 1), nb);
            w[2] = wb * (1.0 - fb);
            w[3] = wb * fb;
        }
        for (int k = 0; k < 4; ++k) {
            pix[k * N + i] = p[k];
            wgt[k * N + i] = w[k];
        }
    }
}

/* RING pix2ang restatement (numba_healpy.py:505-535). */
void oracle_pix2ang(int64_t nside, const int64_t *pixs, int64_t N, double *theta, double *phi) {
    const int64_t npix = 12 * nside * nside;
    const int64_t ncap = 2 * nside * (nside - 1);
    for (int64_t i = 0; i < N; ++i) {
        int64_t pix = pixs[i], iring, ip_in;
        if (pix < ncap) {
            iring = orc_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)pix)));
            ip_in = pix - 2 * iring * (iring - 1);
        } else if (pix < npix - ncap) {
            int64_t ip = pix - ncap;
            iring = ip / (4 * nside) + nside;
            ip_in = ip % (4 * nside);
        } else {
            int64_t ips = npix - pix - 1;
            int64_t irs = orc_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)ips)));
            iring = 4 * nside - irs;
            ip_in = pix - (npix - 2 * irs * (irs + 1));
        }
        int64_t n, fp;
        double phi0, dphi;
        orc_ring_info(nside, iring, npix, &n, &fp, &phi0, &dphi);
        phi[i] = phi0 + (double)ip_in * dphi;
        theta[i] = acos(orc_ring_z(nside, iring));
    }
}

/* RING ang2pix restatement, 4-candidate rule (numba_healpy.py:642-693). */
void oracle_ang2pix(int64_t nside, const double *theta, const double *phi, int64_t N,
                    int64_t *out) {
    const int64_t npix = 12 * nside * nside;
    for (int64_t i = 0; i < N; ++i) {
        double z = cos(theta[i]);
        double phi_w = orc_fmod(phi[i], ORC_TWO_PI);
        int64_t ir_above = orc_ring_above(nside, z);
        if (ir_above < 1)
            ir_above = 1;
        else if (ir_above > 4 * nside - 2)
            ir_above = 4 * nside - 2;
        int64_t best_pix = -1;
        double best_cos = -2.0;
        double sin_th = sin(theta[i]);
        for (int g = 0; g < 2; ++g) {
            int64_t ir = ir_above + g;
            if (ir < 1 || ir > 4 * nside - 1) continue;
            int64_t n, fp;
            double phi0, dphi;
            orc_ring_info(nside, ir, npix, &n, &fp, &phi0, &dphi);
            double zc = orc_ring_z(nside, ir);
            double szc = sqrt(orc_max0(1.0 - zc * zc));
            int64_t ipb = orc_imod(orc_int(phi_w * (double)n / ORC_TWO_PI), n);
            for (int t = 0; t < 2; ++t) {
                int64_t ip = t == 0 ? ipb : orc_imod(ipb + 1, n);
                double phic = phi0 + (double)ip * dphi;
                double cosd = sin_th * szc * cos(phi_w - phic) + z * zc;
                if (cosd > best_cos) {
                    best_cos = cosd;
                    best_pix = fp + ip;
                }
            }
        }
        out[i] = best_pix;
    }
}

/* Scalar spin-2 for tests (tod_bilinear.py:84-145). */
void oracle_spin2(const double *z_pix, const double *sth_pix, const double *phi_pix,
                  const double *z_pts, const double *sth_pts, const double *phi_pts, int64_t N,
                  double *c2d, double *s2d) {
    for (int64_t i = 0; i < N; ++i)
        orc_spin2(z_pix[i], sth_pix[i], phi_pix[i], z_pts[i], sth_pts[i], phi_pts[i], &c2d[i],
                  &s2d[i]);
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
