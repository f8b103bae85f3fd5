// sky_synth.cu -- spherical-harmonic synthesis of a real HEALPix RING map
// (alm -> map) on the GPU, for seeded synthetic skies with a given power
// spectrum.  It stands in for healpy.synfast/alm2map, which the reference's
// benchmark configurations name and which is not available here.
//
// map(theta, phi) = sum_l [ a_l0 L_l0(cos theta)
//                          + 2 sum_{m>0} Re(a_lm L_lm(cos theta) e^{i m phi}) ]
// with the orthonormal associated Legendre functions L_lm (Condon-Shortley
// phase), a_lm stored m-major: index(l, m) = m (2 lmax + 1 - m) / 2 + l.
//
// Stage 1 (legendre_kernel): one thread per (north ring, m) runs the
// three-term recurrence in l
//   L_mm      = (-1)^m sqrt((2m+1)/(4 pi) prod_{k<=m} (2k-1)/(2k)) sin^m theta
//   L_{m+1,m} = x sqrt(2m+3) L_mm
//   L_lm      = a_lm (x L_{l-1,m} - b_lm L_{l-2,m}),
//   a_lm = sqrt((4 l^2 - 1)/(l^2 - m^2)), b_lm = sqrt(((l-1)^2 - m^2)/(4 (l-1)^2 - 1)),
// carrying the value as mantissa * 2^(256 k) so that the tiny starting values
// near the poles do not underflow (terms are accumulated once k reaches 0),
// and uses L_lm(-x) = (-1)^(l+m) L_lm(x) to produce the mirrored south ring.
// Stage 2 (ring_sum_kernel): one thread per pixel sums over m with the
// rotation e^{i m phi} advanced by complex multiplication.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "gather_impl.cuh"

namespace todgpu {

constexpr double kScale = 1.157920892373162e77;     // 2^256
constexpr double kInvScale = 8.636168555094445e-78;  // 2^-256

// F[r][m] (north) and F[rs][m] (mirrored south ring) for rings r = 1..2 nside.
__global__ void legendre_kernel(long long nside, int lmax, const double2* alm, double2* F) {
  const long long nrings_n = 2 * nside;  // rings 1 .. 2 nside (2 nside = equator)
  const long long total = nrings_n * (long long)(lmax + 1);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long r = 1 + t / (lmax + 1);
    const int m = (int)(t % (lmax + 1));
    const double x = hp_ring_z(nside, r);
    const double sinth = sqrt((1.0 - x) * (1.0 + x));
    // log2 |L_mm|: prod_{k<=m} (2k-1)/(2k) = (2m)! / (4^m (m!)^2)
    const double kLog2e = 1.4426950408889634;
    double lg = 0.5 * log2((2.0 * m + 1.0) / (4.0 * kPi)) +
                0.5 * kLog2e * (lgamma(2.0 * m + 1.0) - 2.0 * lgamma(m + 1.0)) - (double)m;
    const double lgs = (sinth > 0.0) ? log2(sinth) : -1e300;
    lg += m * lgs;
    // scale only starting values below the normal double range
    long long ke = 0;
    if (lg < -900.0) ke = (long long)floor((lg + 300.0) / 256.0);
    double v_prev = 0.0;                                     // L_{l-1,m} (scaled)
    double v = exp2(lg - 256.0 * (double)ke) * ((m & 1) ? -1.0 : 1.0);  // L_mm
    if (m > 0 && sinth == 0.0) v = 0.0;
    const long long base = (long long)m * (2LL * lmax + 1 - m) / 2;
    double2 fn = make_double2(0.0, 0.0), fs = make_double2(0.0, 0.0);
    const bool mirror = r < 2 * nside;
    for (int l = m; l <= lmax; ++l) {
      if (l > m) {
        double vn;
        if (l == m + 1) {
          vn = x * sqrt(2.0 * m + 3.0) * v;
        } else {
          const double l2 = (double)l * l, m2 = (double)m * m, lm1 = (double)(l - 1);
          const double a = sqrt((4.0 * l2 - 1.0) / (l2 - m2));
          const double b = sqrt((lm1 * lm1 - m2) / (4.0 * lm1 * lm1 - 1.0));
          vn = a * (x * v - b * v_prev);
        }
        v_prev = v;
        v = vn;
        if (ke < 0 && fabs(v) > kScale) {
          v *= kInvScale;
          v_prev *= kInvScale;
          ++ke;
        }
      }
      if (ke == 0) {
        const double2 c = alm[base + l];
        fn.x += c.x * v;
        fn.y += c.y * v;
        if (mirror) {
          const double sgn = ((l + m) & 1) ? -1.0 : 1.0;
          fs.x += sgn * c.x * v;
          fs.y += sgn * c.y * v;
        }
      }
    }
    F[(r - 1) * (lmax + 1) + m] = fn;
    if (mirror) F[(4 * nside - 1 - r) * (lmax + 1) + m] = fs;
  }
}

// map[p] = F_0 + 2 sum_{m >= 1} Re(F_m e^{i m phi_p}) for the pixel's ring.
__global__ void ring_sum_kernel(long long nside, int lmax, const double2* F, double* out, long long out_stride,
                                int comp) {
  const long long npix = 12 * nside * nside;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix;
       p += (long long)gridDim.x * blockDim.x) {
    // ring of pixel p
    const long long ncap = 2 * nside * (nside - 1);
    long long ir, ip;
    if (p < ncap) {
      ir = py_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)p)));
      if (2 * ir * (ir - 1) > p) --ir;
      if (2 * (ir + 1) * ir <= p) ++ir;
      ip = p - 2 * ir * (ir - 1);
    } else if (p < npix - ncap) {
      const long long q = p - ncap;
      ir = q / (4 * nside) + nside;
      ip = q % (4 * nside);
    } else {
      const long long ps = npix - p - 1;
      long long irs = py_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)ps)));
      if (2 * irs * (irs - 1) > ps) --irs;
      if (2 * (irs + 1) * irs <= ps) ++irs;
      ir = 4 * nside - irs;
      ip = p - (npix - 2 * irs * (irs + 1));
    }
    const RingInfo ri = hp_ring_info(nside, ir, npix);
    const double phi = ri.phi0 + (double)ip * ri.dphi;
    double s1, c1;
    sincos(phi, &s1, &c1);
    const double2* f = F + (ir - 1) * (lmax + 1);
    double acc = f[0].x;
    double cr = c1, ci = s1;  // e^{i m phi}, m = 1
    for (int m = 1; m <= lmax; ++m) {
      const double2 fm = f[m];
      acc += 2.0 * (fm.x * cr - fm.y * ci);
      if ((m & 63) == 0) {
        sincos((double)(m + 1) * phi, &ci, &cr);  // re-anchor e^{i (m+1) phi}
      } else {
        const double nr = cr * c1 - ci * s1;
        ci = cr * s1 + ci * c1;
        cr = nr;
      }
    }
    out[(long long)comp * out_stride + p] = acc;
  }
}

}  // namespace todgpu

using namespace todgpu;

extern "C" size_t todgpu_alm2map_workspace_bytes(int64_t nside, int32_t lmax) {
  if (nside < 1 || nside > kMaxNside || lmax < 0) return 0;
  return sizeof(double2) * (size_t)(4 * nside - 1) * (size_t)(lmax + 1);
}

extern "C" int todgpu_alm2map(int64_t nside, int32_t lmax, const void* alm, void* workspace, size_t ws_bytes,
                              double* map, int64_t map_stride, int32_t comp, void* stream) {
  if (nside < 1 || nside > kMaxNside) return fail(TODGPU_ENSIDE, "nside out of range");
  if (lmax < 0 || lmax > 4 * nside) return fail(TODGPU_ESHAPE, "lmax out of range");
  if (!alm || !workspace || !map) return fail(TODGPU_EINVAL, "NULL pointer");
  if (ws_bytes < todgpu_alm2map_workspace_bytes(nside, lmax)) return fail(TODGPU_ESHAPE, "workspace too small");
  if (map_stride < 12 * nside * nside || comp < 0) return fail(TODGPU_ESHAPE, "bad map stride or component");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double2* F = static_cast<double2*>(workspace);
  const long long jobs = 2 * nside * (long long)(lmax + 1);
  legendre_kernel<<<(unsigned)std::min<long long>((jobs + 127) / 128, 148LL * 64), 128, 0, s>>>(
      nside, lmax, static_cast<const double2*>(alm), F);
  const long long npix = 12 * nside * nside;
  ring_sum_kernel<<<(unsigned)std::min<long long>((npix + 255) / 256, 148LL * 64), 256, 0, s>>>(nside, lmax, F, map,
                                                                                              map_stride, comp);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "alm2map kernels");
}
