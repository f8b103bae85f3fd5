// healpix_ring.cuh -- device-side HEALPix RING geometry, bilinear stencil,
// nearest-pixel search, spin-2 frame rotation and the double Rodrigues
// rotation of the beam-convolution TOD path.
//
// Every function reproduces the decisions of the reference implementation
// (ArtemBasyrov/tod_generation_mapbased_beam) exactly: same operation order,
// same operand types, Python float-modulo semantics and x86 int() truncation.
// The translation units that include this header are compiled with
// -fmad=false so that no multiply-add is contracted (the reference's Numba
// code is not contracted either); helpers that want a fused multiply-add call
// fma()/fmaf() explicitly.
//
//   numba_healpy.py:53-70    ring_above      -> hp_ring_above
//   numba_healpy.py:73-101   ring_info       -> hp_ring_info
//   numba_healpy.py:104-114  ring_z          -> hp_ring_z
//   numba_healpy.py:358-499  ring interp     -> hp_stencil
//   numba_healpy.py:642-693  ang2pix rule    -> hp_nearest
//   tod_rotations.py:83-134  Rodrigues       -> rot_ref32 / rot_f64
//   tod_bilinear.py:84-145   spin-2          -> spin2_c2s2
#pragma once

#include <cstdint>
#include <math.h>

namespace todgpu {

constexpr double kPi = 3.141592653589793;
constexpr double kTwoPi = 2.0 * 3.141592653589793;
constexpr double kTwoThirds = 2.0 / 3.0;

// int(x) of a float64 as x86 cvttsd2si computes it: NaN or out-of-range
// values give INT64_MIN.
__device__ __forceinline__ long long py_int(double x) {
  if (!(x >= -9223372036854775808.0 && x < 9223372036854775808.0)) return (long long)0x8000000000000000ULL;
  return __double2ll_rz(x);
}

// Python `x % w` for floats with w > 0 (CPython float_rem semantics).  The
// quotient operands on this path satisfy |x| < w except at exact ring ends,
// where fmod takes over.
__device__ __forceinline__ double py_fmod_pos(double x, double w) {
  double m = (fabs(x) < w) ? x : fmod(x, w);
  if (m != 0.0) {
    if (m < 0.0) m = m + w;
  } else {
    m = 0.0;
  }
  return m;
}

// Python `a % n` for integers, n > 0, with a fast path for 0 <= a < 2n.
__device__ __forceinline__ long long py_imod(long long a, long long n) {
  if (a >= 0 && a < n) return a;
  if (a >= n && a < 2 * n) return a - n;
  long long r = a % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ long long wrap_add(long long a, long long b) {
  return (long long)((unsigned long long)a + (unsigned long long)b);
}

__device__ __forceinline__ double max0(double x) { return x > 0.0 ? x : 0.0; }
__device__ __forceinline__ double clamp1(double x) {
  double a = (x < 1.0) ? x : 1.0;
  return (a > -1.0) ? a : -1.0;
}

// theta_q - theta_a for a query z and a nearby ring (z_a, s_a = sin theta_a):
// sin(theta_q - theta_a) = z_a sin(theta_q) - z sin(theta_a), and for |d| <
// 0.01 asin(d) = d + d^3/6 + 3 d^5/40 + 5 d^7/112 (the next term is below
// 3e-20).  Returns false when the angle is too large for the series.
__device__ __forceinline__ bool dtheta_small(double z, double za, double sa, double& out) {
  const double sq = sqrt((1.0 - z) * (1.0 + z));
  const double d = fma(za, sq, -z * sa);
  if (!(fabs(d) < 0.01)) return false;
  const double d2 = d * d;
  out = fma(d * d2, fma(d2, fma(d2, 5.0 / 112.0, 3.0 / 40.0), 1.0 / 6.0), d);
  return true;
}

// Index of the last ring whose centre z is > z (1-based; 0 above ring 1).
__device__ __forceinline__ long long hp_ring_above(long long nside, double z) {
  double az = fabs(z);
  long long ir;
  if (az > kTwoThirds) {
    double tp = (double)nside * sqrt(3.0 * (1.0 - az));
    ir = py_int(tp);
    if (z < 0.0) ir = wrap_add(wrap_add(4 * nside, -ir), -1);
  } else {
    ir = py_int((double)nside * (2.0 - 1.5 * z));
  }
  return ir;
}

struct RingInfo {
  long long n;      // pixels in the ring
  long long first;  // first pixel index
  double phi0;      // longitude of the first pixel
  double dphi;      // pixel spacing
};

__device__ __forceinline__ RingInfo hp_ring_info(long long nside, long long ir, long long npix) {
  RingInfo r;
  long long s;
  if (ir < nside) {
    r.n = 4 * ir;
    r.first = 2 * ir * (ir - 1);
    s = 1;
  } else if (ir <= 3 * nside) {
    r.n = 4 * nside;
    r.first = 2 * nside * (nside - 1) + (ir - nside) * 4 * nside;
    s = (((ir - nside) & 1) == 0) ? 1 : 0;
  } else {
    long long i2 = 4 * nside - ir;
    r.n = 4 * i2;
    r.first = npix - 2 * i2 * (i2 + 1);
    s = 1;
  }
  r.dphi = kTwoPi / (double)r.n;
  r.phi0 = (double)s * r.dphi * 0.5;
  return r;
}

__device__ __forceinline__ double hp_ring_z(long long nside, long long ir) {
  if (ir < nside) {
    double t = (double)ir;
    return 1.0 - t * t / (3.0 * (double)nside * (double)nside);
  } else if (ir <= 3 * nside) {
    return kTwoThirds * (2.0 - (double)ir / (double)nside);
  } else {
    double t = (double)(4 * nside - ir);
    return -(1.0 - t * t / (3.0 * (double)nside * (double)nside));
  }
}

// Everything the stencil needs about one ring.  `ta` is acos(z).
struct RingData {
  long long n, first;
  double phi0, dphi, z, ta;
};

// Ring provider that derives every ring quantity on the fly.
struct DirectRings {
  long long nside, npix;
  __device__ __forceinline__ RingData operator()(long long ir) const {
    RingInfo r = hp_ring_info(nside, ir, npix);
    RingData d;
    d.n = r.n;
    d.first = r.first;
    d.phi0 = r.phi0;
    d.dphi = r.dphi;
    d.z = hp_ring_z(nside, ir);
    d.ta = acos(d.z);
    return d;
  }
  __device__ __forceinline__ double sth(long long, const RingData& d) const { return sqrt(max0(1.0 - d.z * d.z)); }
};

// Ring provider for the nearest rule, which needs no acos of the ring z.
struct DirectRingsNoAcos {
  long long nside, npix;
  __device__ __forceinline__ RingData operator()(long long ir) const {
    RingInfo r = hp_ring_info(nside, ir, npix);
    RingData d;
    d.n = r.n;
    d.first = r.first;
    d.phi0 = r.phi0;
    d.dphi = r.dphi;
    d.z = hp_ring_z(nside, ir);
    d.ta = 0.0;
    return d;
  }
  __device__ __forceinline__ double sth(long long, const RingData& d) const { return sqrt(max0(1.0 - d.z * d.z)); }
};

// 4-neighbour bilinear stencil of a query (z clamped to [-1,1], phi in
// [0, 2pi)).  For each neighbour k = 0..3, in the reference's order, calls
//   visit(k, pixel, weight, ring, in_ring_index, ring_length, ring_z, pixel_phi)
// The in-ring index equals the ring length n when the reference's phi modulo
// rounds up to n: the pixel then spills into the next ring, exactly as in the
// reference (numba_healpy.py:453-471).
template <class Rings, class Visit>
__device__ __forceinline__ void hp_stencil(long long nside, double z, double phi_w, const Rings& rings,
                                           Visit&& visit) {
  const long long ir_above = hp_ring_above(nside, z);
  const long long ir_below = wrap_add(ir_above, 1);
  if (ir_above == 0) {
    // North of ring 1: ring 1 pair plus the opposite pair of ring 1.
    const RingData ra = rings(1);
    const double tw = py_fmod_pos((phi_w - ra.phi0) / ra.dphi, (double)ra.n);
    const long long ip = py_int(tw);
    const double frac = tw - (double)ip;
    const long long ip2 = py_imod(wrap_add(ip, 1), ra.n);
    const long long o1 = py_imod(wrap_add(ip, 2), ra.n), o2 = py_imod(ip2 + 2, ra.n);
    const double theta = acos(z);
    const double wt = theta / ra.ta;
    const double nf = (1.0 - wt) * 0.25;
    visit(0, ra.first + o1, nf, 1LL, o1, ra.n, ra.z, ra.phi0 + (double)o1 * ra.dphi);
    visit(1, ra.first + o2, nf, 1LL, o2, ra.n, ra.z, ra.phi0 + (double)o2 * ra.dphi);
    visit(2, wrap_add(ra.first, ip), (1.0 - frac) * wt + nf, 1LL, ip, ra.n, ra.z, ra.phi0 + (double)ip * ra.dphi);
    visit(3, ra.first + ip2, frac * wt + nf, 1LL, ip2, ra.n, ra.z, ra.phi0 + (double)ip2 * ra.dphi);
  } else if (ir_below == 4 * nside) {
    // South of the last ring: last-ring pair plus its opposite pair.
    const long long ir_last = 4 * nside - 1;
    const RingData ra = rings(ir_last);
    const double tw = py_fmod_pos((phi_w - ra.phi0) / ra.dphi, (double)ra.n);
    const long long ip = py_int(tw);
    const double frac = tw - (double)ip;
    const long long ip2 = py_imod(wrap_add(ip, 1), ra.n);
    const long long o1 = py_imod(wrap_add(ip, 2), ra.n), o2 = py_imod(ip2 + 2, ra.n);
    const double theta = acos(z);
    const double ws = (theta - ra.ta) / (kPi - ra.ta);
    const double sf = ws * 0.25;
    visit(0, wrap_add(ra.first, ip), (1.0 - frac) * (1.0 - ws) + sf, ir_last, ip, ra.n, ra.z,
          ra.phi0 + (double)ip * ra.dphi);
    visit(1, ra.first + ip2, frac * (1.0 - ws) + sf, ir_last, ip2, ra.n, ra.z, ra.phi0 + (double)ip2 * ra.dphi);
    visit(2, ra.first + o1, sf, ir_last, o1, ra.n, ra.z, ra.phi0 + (double)o1 * ra.dphi);
    visit(3, ra.first + o2, sf, ir_last, o2, ra.n, ra.z, ra.phi0 + (double)o2 * ra.dphi);
  } else {
    const RingData ra = rings(ir_above);
    const RingData rb = rings(ir_below);
    double dta;
    if (!dtheta_small(z, ra.z, rings.sth(ir_above, ra), dta)) dta = acos(z) - ra.ta;
    const double wb = dta / (rb.ta - ra.ta);
    const double wa = 1.0 - wb;
    double tw = py_fmod_pos((phi_w - ra.phi0) / ra.dphi, (double)ra.n);
    const long long ia = py_int(tw);
    const double fa = tw - (double)ia;
    const long long ia1 = py_imod(wrap_add(ia, 1), ra.n);
    visit(0, wrap_add(ra.first, ia), wa * (1.0 - fa), ir_above, ia, ra.n, ra.z, ra.phi0 + (double)ia * ra.dphi);
    visit(1, ra.first + ia1, wa * fa, ir_above, ia1, ra.n, ra.z, ra.phi0 + (double)ia1 * ra.dphi);
    tw = py_fmod_pos((phi_w - rb.phi0) / rb.dphi, (double)rb.n);
    const long long ib = py_int(tw);
    const double fb = tw - (double)ib;
    const long long ib1 = py_imod(wrap_add(ib, 1), rb.n);
    visit(2, wrap_add(rb.first, ib), wb * (1.0 - fb), ir_below, ib, rb.n, rb.z, rb.phi0 + (double)ib * rb.dphi);
    visit(3, rb.first + ib1, wb * fb, ir_below, ib1, rb.n, rb.z, rb.phi0 + (double)ib1 * rb.dphi);
  }
}

// Nearest pixel by the reference's 4-candidate rule (two rings bracketing z,
// two phi slots per ring, maximum cos distance; ties keep the first).
// z and sin_th are used as given (the nearest kernel passes the unnormalised
// rotated z and sqrt(vx^2+vy^2)).  `ring_sth(ir, d)` returns
// sqrt(max(0, 1 - z_ring^2)) for ring data d.
struct Nearest {
  long long pix;
  long long ring;
  long long ip;  // in-ring index, always in [0, n)
  long long n;   // pixels in the chosen ring
  double zc;
  double phic;
};

template <class Rings>
__device__ __forceinline__ Nearest hp_nearest(long long nside, double z, double sin_th, double phi_w,
                                              const Rings& rings) {
  long long ir_above = hp_ring_above(nside, z);
  if (ir_above < 1)
    ir_above = 1;
  else if (ir_above > 4 * nside - 2)
    ir_above = 4 * nside - 2;
  Nearest best;
  best.pix = 0;
  best.ring = 0;
  best.ip = 0;
  best.n = 1;
  best.zc = 0.0;
  best.phic = 0.0;
  double best_cos = -2.0;
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    const long long ir = ir_above + g;
    const RingData r = rings(ir);
    const double szc = rings.sth(ir, r);
    const long long ipb = py_imod(py_int(phi_w * (double)r.n / kTwoPi), r.n);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const long long ip = (t == 0) ? ipb : py_imod(ipb + 1, r.n);
      const double phic = r.phi0 + (double)ip * r.dphi;
      const double cosd = sin_th * szc * cos(phi_w - phic) + z * r.z;
      if (cosd > best_cos) {
        best_cos = cosd;
        best.pix = r.first + ip;
        best.ring = ir;
        best.ip = ip;
        best.n = r.n;
        best.zc = r.z;
        best.phic = phic;
      }
    }
  }
  return best;
}

// cos 2d, sin 2d of the frame rotation between a pixel centre and the
// boresight (tan d = N/D from the haversine form; identity for equal points),
// tod_bilinear.py:84-145.  Evaluated in the reference's exact operation order
// (no contraction): near the poles D is a difference of nearly equal terms,
// so any reassociation moves the result by far more than an ulp.
__device__ __forceinline__ void spin2_c2s2(double z_pix, double sth_pix, double phi_pix, double z_pts,
                                           double sth_pts, double phi_pts, double& c2d, double& s2d) {
  if (phi_pts == phi_pix && sth_pts == sth_pix && z_pts == z_pix) {
    c2d = 1.0;
    s2d = 0.0;
    return;
  }
  const double dphi = phi_pts - phi_pix;
  double sh, ch;
  sincos(dphi * 0.5, &sh, &ch);
  const double sin_dphi = 2.0 * ch * sh;
  const double cos_dphi = 1.0 - 2.0 * sh * sh;
  const double sh2 = sh * sh;
  const double dz = z_pts - z_pix;
  const double ds = sth_pts - sth_pix;
  const double st2 = 0.25 * (dz * dz + ds * ds);
  const double S = sth_pix * sth_pts;
  const double h = st2 + S * sh2;
  const double sin2_dtheta = 4.0 * st2 * (1.0 - st2);
  const double z_sum = z_pts + z_pix;
  const double N = 2.0 * sin_dphi * z_sum * h;
  const double C = z_pts * z_pix;
  const double term1 = sin2_dtheta * cos_dphi;
  const double term2 = 4.0 * S * C * sh2 * sh2;
  const double term3 = S * sin_dphi * sin_dphi;
  const double D = term1 - term2 + term3;
  const double u = 1.0 / (N * N + D * D);
  c2d = (D * D - N * N) * u;
  s2d = 2.0 * N * D * u;
}

// Per-sample rotation: recentre about axis k by angle a, then roll about the
// boresight p by angle psi.
struct SampleRot {
  double kx, ky, kz, ca, sa, px, py, pz, cp, sp;  // float64 form
  float fkx, fky, fkz, fca, fsa;                  // float32 recentre inputs
};

// Reference operand typing (float32 parameters read through float(), which
// Numba keeps float32): the recentre products and sums are float32, the
// (1 - cos) factor and the roll are float64.
__device__ __forceinline__ void rot_ref32(const SampleRot& r, float vx, float vy, float vz, double& ox,
                                          double& oy, double& oz) {
  const double oma = 1.0 - (double)r.fca;
  const double omp = 1.0 - r.cp;
  const float dkv = r.fkx * vx + r.fky * vy + r.fkz * vz;
  const float ax = vx * r.fca + (r.fky * vz - r.fkz * vy) * r.fsa;
  const float ay = vy * r.fca + (r.fkz * vx - r.fkx * vz) * r.fsa;
  const float az = vz * r.fca + (r.fkx * vy - r.fky * vx) * r.fsa;
  const double rx = (double)ax + (double)(r.fkx * dkv) * oma;
  const double ry = (double)ay + (double)(r.fky * dkv) * oma;
  const double rz = (double)az + (double)(r.fkz * dkv) * oma;
  const double dpr = r.px * rx + r.py * ry + r.pz * rz;
  ox = rx * r.cp + (r.py * rz - r.pz * ry) * r.sp + r.px * dpr * omp;
  oy = ry * r.cp + (r.pz * rx - r.px * rz) * r.sp + r.py * dpr * omp;
  oz = rz * r.cp + (r.px * ry - r.py * rx) * r.sp + r.pz * dpr * omp;
}

// All-float64 rotation (precision form / ideal oracle semantics).
__device__ __forceinline__ void rot_f64(const SampleRot& r, double vx, double vy, double vz, double& ox,
                                        double& oy, double& oz) {
  const double oma = 1.0 - r.ca;
  const double omp = 1.0 - r.cp;
  const double dkv = r.kx * vx + r.ky * vy + r.kz * vz;
  const double rx = vx * r.ca + (r.ky * vz - r.kz * vy) * r.sa + r.kx * dkv * oma;
  const double ry = vy * r.ca + (r.kz * vx - r.kx * vz) * r.sa + r.ky * dkv * oma;
  const double rz = vz * r.ca + (r.kx * vy - r.ky * vx) * r.sa + r.kz * dkv * oma;
  const double dpr = r.px * rx + r.py * ry + r.pz * rz;
  ox = rx * r.cp + (r.py * rz - r.pz * ry) * r.sp + r.px * dpr * omp;
  oy = ry * r.cp + (r.pz * rx - r.px * rz) * r.sp + r.py * dpr * omp;
  oz = rz * r.cp + (r.px * ry - r.py * rx) * r.sp + r.pz * dpr * omp;
}

}  // namespace todgpu
