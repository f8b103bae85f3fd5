// gather_impl.cuh -- fused beam-convolution TOD kernels for B200 (sm_100a):
// device code and launch templates, shared by the translation units that
// instantiate them (gather_map_*.cu, one per map element type) and by the C
// ABI (tod_api.cu).
//
// Work decomposition ("footprint" kernel): a persistent grid of CTAs (128
// threads, 8 per SM, when the sample's spin-2 table fits an eighth of an SM's
// shared memory; else 256 threads, 3-4 per SM) walks the samples; a CTA takes
// one sample at a time and
//   1. rotates the beam's centre direction with the sample's rotation to get
//      the footprint centre, and derives the window of RING rings the
//      footprint (beam radius + stencil reach) can touch;
//   2. tabulates per window ring (in shared memory) the ring layout, ring z,
//      acos(ring z) and sqrt(1 - z^2), and the longitude range of ring pixels
//      inside the footprint;
//   3. tabulates cos 2d / sin 2d of the spin-2 frame rotation for every ring
//      pixel in the footprint once (a stencil pixel is shared by ~16 (beam
//      pixel, neighbour) pairs of a sample);
//   4. strides its threads over the beam pixels: rotate -> atan2/clamp ->
//      RING stencil (ring data from the window) -> spin-2 (from the table) ->
//      gather -> FP64 accumulate;
//   5. reduces the per-lane sums (256 summation lanes in either CTA shape) in
//      a fixed order and adds them into tod[c, b] (one writer per sample: no
//      atomics, bit-reproducible runs, the same TOD in both shapes).
// Table values are produced by the same functions on the same inputs as
// direct evaluation, so they are bit-identical to it; any lookup outside the
// window (or a footprint too large for the tables) falls back to direct
// evaluation.  The window therefore only decides speed, never results.
//
// Compiled with -fmad=false: the pixel decisions and the FP64 accumulation
// reproduce the reference's uncontracted arithmetic.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "healpix_ring.cuh"
#include "todgpu.h"

namespace todgpu {

constexpr int kRingCap = 192;   // rings per footprint window
constexpr int kTabCapDefault = 2048;  // spin-2 table slots per sample (32 KB)
constexpr long long kMaxNside = 16384;
constexpr int kNTStatic = 256;  // threads of the reach kernel of the built-in table
// Summation lanes of the gather: the beam pixels of a sample are summed in
// kSumLanes strided partial sums (then per warp of lanes, then over those in
// order), whatever the CTA's thread count, so CTAs of 128 and 256 threads
// give the same TOD bit for bit.
constexpr int kSumLanes = 256;
// The narrow CTA shape (128 threads, 8 per SM) and the window rings its table
// header always reserves, so that the table's offset is a compile-time constant
// of that shape (the wide shape sizes its header per launch).
constexpr int kNTNarrow = 128;
constexpr int kMinbNarrow = 8;
constexpr int kRingCapNarrow = 80;

// Message of the calling thread's last failure (defined in tod_api.cu).
extern thread_local std::string g_last_error;

inline int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

inline int cuda_fail(cudaError_t e, const char* what) {
  return fail(TODGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct KArgs {
  long long nside, npix, B, S;
  int C, c_q, c_u;
  int tab_cap;               // spin-2 table slots in shared memory
  int tab_req;               // slots the caller asks for (0: default)
  const void* ring_table;    // RingRec[4 nside] or nullptr
  const void* vec;
  const void* axes;
  const void* cos_a;
  const void* sin_a;
  const void* pts;
  const void* cos_p;
  const void* sin_p;
  const float* bore_phi;
  const void* theta;         // pointing angles (angles mode)
  const void* phi;
  const void* psi;
  int angles_f32;            // angles are float32 (else float64)
  double cvx, cvy, cvz;      // beam-centre unit vector (angles mode)
  double cnx, cny, cnz;      // its local north
  const float* beam;
  const void* map;
  long long map_stride;
  double* tod;
  long long tod_stride;
  unsigned long long* err;
  int flags_stage;           // the caller allows staging the beam in shared memory
  int beam_stage;            // the launch made room for the beam in shared memory
  int flags_wide;            // the caller asks for 256-thread CTAs
  int ring_cap;              // window rings the launch's table header holds
};

// Pointing modes of the per-sample rotation.
constexpr int kParamsRef32 = 0;  // reference float32 parameter arrays
constexpr int kParamsF64 = 1;    // float64 parameter arrays
constexpr int kAngles = 2;       // (theta, phi, psi) + beam centre, derived on the device

__host__ __device__ constexpr bool f64_params(int pm) { return pm == kParamsF64; }

template <int PM>
__device__ __forceinline__ double angle_at(const KArgs& a, const void* p, long long b) {
  return a.angles_f32 ? (double)static_cast<const float*>(p)[b] : static_cast<const double*>(p)[b];
}

// Rotation from pointing angles (theta, phi, psi), in float64: the Rodrigues
// vector taking the beam centre c to the boresight t and the polarisation
// offset beta (tod_rotations.py:219-303), then the parameters of
// tod_rotations.py:306-333 without any float32 rounding.
__device__ __forceinline__ SampleRot rot_from_angle_values(const KArgs& a, double th, double ph, double ps) {
  double st, ct, sp, cp;
  sincos(th, &st, &ct);
  sincos(ph, &sp, &cp);
  const double tx = st * cp, ty = st * sp, tz = ct;    // boresight
  const double nx = cp * ct, ny = sp * ct, nz = -st;   // its north
  const double ex = -sp, ey = cp;                      // its east
  double kx = a.cvy * tz - a.cvz * ty;
  double ky = a.cvz * tx - a.cvx * tz;
  double kz = a.cvx * ty - a.cvy * tx;
  const double kn = sqrt((kx * kx + ky * ky) + kz * kz);
  if (kn > 1e-10) {
    kx /= kn;
    ky /= kn;
    kz /= kn;
  } else {
    kx = ky = kz = 0.0;
  }
  const double ang = acos(clamp1(a.cvx * tx + a.cvy * ty + a.cvz * tz));
  double sa, ca;
  sincos(ang, &sa, &ca);
  const double dkn = kx * a.cnx + ky * a.cny + kz * a.cnz;
  const double oma = 1.0 - ca;
  const double wx = a.cnx * ca + (ky * a.cnz - kz * a.cny) * sa + kx * dkn * oma;
  const double wy = a.cny * ca + (kz * a.cnx - kx * a.cnz) * sa + ky * dkn * oma;
  const double wz = a.cnz * ca + (kx * a.cny - ky * a.cnx) * sa + kz * dkn * oma;
  double beta = atan2(wx * ex + wy * ey + wz * 0.0, wx * nx + wy * ny + wz * nz);
  if (beta < 0.0) beta += kTwoPi;
  SampleRot r;
  r.kx = kx;
  r.ky = ky;
  r.kz = kz;
  r.ca = ca;
  r.sa = sa;
  r.px = tx;
  r.py = ty;
  r.pz = tz;
  sincos(ps - beta, &r.sp, &r.cp);
  return r;
}

__device__ __forceinline__ SampleRot rot_from_angles(const KArgs& a, long long b) {
  return rot_from_angle_values(a, angle_at<kAngles>(a, a.theta, b), angle_at<kAngles>(a, a.phi, b),
                               angle_at<kAngles>(a, a.psi, b));
}

// The per-sample pointing inputs as numbered fields.  Reference float32
// parameters: 0-2 axes, 3 cos_a, 4 sin_a, 5-7 ax_pts, 8 cos_p, 9 sin_p, 10 the
// boresight longitude (when given); float64 parameters: fields 0-9 as
// doubles; angles: 0 theta, 1 phi, 2 psi.  field_ptr gives a field's address
// (nullptr when absent), field_bytes its size.
template <int PM>
__device__ __forceinline__ const void* field_ptr(const KArgs& a, long long b, int i) {
  if constexpr (PM == kAngles) {
    const void* p = i == 0 ? a.theta : (i == 1 ? a.phi : a.psi);
    return a.angles_f32 ? (const void*)(static_cast<const float*>(p) + b)
                        : (const void*)(static_cast<const double*>(p) + b);
  } else {
    using T = typename std::conditional<PM == kParamsRef32, float, double>::type;
    if (i < 3) return static_cast<const T*>(a.axes) + 3 * b + i;
    if (i == 3) return static_cast<const T*>(a.cos_a) + b;
    if (i == 4) return static_cast<const T*>(a.sin_a) + b;
    if (i < 8) return static_cast<const T*>(a.pts) + 3 * b + (i - 5);
    if (i == 8) return static_cast<const T*>(a.cos_p) + b;
    if (i == 9) return static_cast<const T*>(a.sin_p) + b;
    if (PM == kParamsRef32 && i == 10 && a.bore_phi != nullptr) return a.bore_phi + b;
    return nullptr;
  }
}
template <int PM>
__device__ __forceinline__ int field_count() {
  return PM == kAngles ? 3 : (PM == kParamsRef32 ? 11 : 10);
}
template <int PM>
__device__ __forceinline__ int field_bytes(const KArgs& a) {
  return PM == kParamsRef32 ? 4 : (PM == kAngles && a.angles_f32 ? 4 : 8);
}

// Rotation of a sample from its fields, got(i) returning field i (float for
// the reference typing, double otherwise).
template <int PM, class Get>
__device__ __forceinline__ SampleRot rot_from_fields(const KArgs& a, const Get& got) {
  SampleRot r;
  if constexpr (PM == kAngles) {
    r = rot_from_angle_values(a, got(0), got(1), got(2));
  } else if constexpr (f64_params(PM)) {
    r.kx = got(0);
    r.ky = got(1);
    r.kz = got(2);
    r.ca = got(3);
    r.sa = got(4);
    r.px = got(5);
    r.py = got(6);
    r.pz = got(7);
    r.cp = got(8);
    r.sp = got(9);
  } else {
    r.fkx = got(0);
    r.fky = got(1);
    r.fkz = got(2);
    r.fca = got(3);
    r.fsa = got(4);
    r.kx = (double)r.fkx;
    r.ky = (double)r.fky;
    r.kz = (double)r.fkz;
    r.ca = (double)r.fca;
    r.sa = (double)r.fsa;
    r.px = (double)got(5);
    r.py = (double)got(6);
    r.pz = (double)got(7);
    r.cp = (double)got(8);
    r.sp = (double)got(9);
  }
  return r;
}

// Boresight (z, sin theta, phi) of the spin-2 angle.  Float32 parameters use
// the reference's typing: sin theta from a float32 square, phi from float32
// atan2 (host libm value when provided).
template <int PM, class Get>
__device__ __forceinline__ void boresight_from_fields(const KArgs& a, const SampleRot& rot, const Get& got, double& z,
                                                      double& sth, double& phi) {
  if constexpr (PM == kAngles) {
    z = clamp1(rot.pz);
    sth = sqrt(max0(1.0 - rot.pz * rot.pz));
    phi = atan2(rot.py, rot.px);
  } else if constexpr (f64_params(PM)) {
    const double pz = got(7);
    z = clamp1(pz);
    sth = sqrt(max0(1.0 - pz * pz));
    phi = atan2((double)got(6), (double)got(5));
  } else {
    const float bz = got(7);
    const float bz2 = bz * bz;
    z = clamp1((double)bz);
    sth = sqrt(max0(1.0 - (double)bz2));
    if (a.bore_phi != nullptr)
      phi = (double)got(10);
    else
      phi = (double)(float)atan2((double)got(6), (double)got(5));
  }
  if (phi < 0.0) phi += kTwoPi;
}

// Field getter reading global memory.
template <int PM>
struct GlobalFields {
  const KArgs& a;
  long long b;
  __device__ __forceinline__ auto operator()(int i) const {
    if constexpr (PM == kParamsRef32)
      return *static_cast<const float*>(field_ptr<PM>(a, b, i));
    else if constexpr (PM == kAngles)
      return a.angles_f32 ? (double)*static_cast<const float*>(field_ptr<PM>(a, b, i))
                          : *static_cast<const double*>(field_ptr<PM>(a, b, i));
    else
      return *static_cast<const double*>(field_ptr<PM>(a, b, i));
  }
};

template <int PM>
__device__ __forceinline__ SampleRot load_rot(const KArgs& a, long long b) {
  return rot_from_fields<PM>(a, GlobalFields<PM>{a, b});
}

template <int PM>
__device__ __forceinline__ void load_boresight(const KArgs& a, const SampleRot& rot, long long b, double& z,
                                               double& sth, double& phi) {
  boresight_from_fields<PM>(a, rot, GlobalFields<PM>{a, b}, z, sth, phi);
}

struct PackF32;
struct PackBF16;
struct PackF64;
template <typename MapT>
__device__ __forceinline__ float4 load_rec(const KArgs& a, long long p);
__device__ __forceinline__ float rec_at(const float4& r, int c);

template <typename MapT>
__device__ __forceinline__ double map_at(const KArgs& a, int c, long long p) {
  if constexpr (std::is_same<MapT, PackF32>::value || std::is_same<MapT, PackBF16>::value)
    return (double)rec_at(load_rec<MapT>(a, p), c);
  else if constexpr (std::is_same<MapT, PackF64>::value)
    return __ldg(static_cast<const double*>(a.map) + 4 * p + c);
  else
    return (double)__ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
}

// mp[c, p] * bv with the nearest kernel's typing (tod_nearest.py:146, :158):
// a float32 map element times the float32 weight is a float32 product.
template <typename MapT>
__device__ __forceinline__ double map_x_beam(const KArgs& a, int c, long long p, float bv) {
  if constexpr (std::is_same<MapT, PackF32>::value || std::is_same<MapT, PackBF16>::value) {
    return (double)(rec_at(load_rec<MapT>(a, p), c) * bv);
  } else if constexpr (std::is_same<MapT, PackF64>::value) {
    return __ldg(static_cast<const double*>(a.map) + 4 * p + c) * (double)bv;
  } else {
    const MapT m = __ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
    if constexpr (sizeof(MapT) == 4)
      return (double)(m * bv);
    else
      return m * (double)bv;
  }
}

// ---------------------------------------------------------------------------
// Map element types.  Planar float/double maps are the reference's
// mp_stacked (C, N); the precision form packs a pixel's components into one
// record: PackF32 = 4 x float32 (16 B), PackBF16 = 4 x bfloat16 (8 B).  The
// precision form also keeps cos 2d / sin 2d in float32 and accumulates in
// float32 with Kahan compensation; pixel decisions and weights stay float64.
// PackF64 = 4 x float64 (32 B, one sector) is the float64 path's layout with
// a pixel's components together: every value and operation as for a planar
// float64 map, so the results are the same bit for bit.
// ---------------------------------------------------------------------------

struct PackF32 {};
struct PackBF16 {};
struct PackF64 {};

template <typename MapT>
struct MapTraits {
  static constexpr bool packed = false;
  using Tab = double2;
};
template <>
struct MapTraits<PackF32> {
  static constexpr bool packed = true;
  using Tab = float2;
};
template <>
struct MapTraits<PackBF16> {
  static constexpr bool packed = true;
  using Tab = float2;
};

__device__ __forceinline__ float bf16_lo(unsigned v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(unsigned v) { return __uint_as_float(v & 0xffff0000u); }

template <typename MapT>
__device__ __forceinline__ float4 load_rec(const KArgs& a, long long p) {
  if constexpr (std::is_same<MapT, PackF32>::value) {
    return __ldg(static_cast<const float4*>(a.map) + p);
  } else {
    const uint2 r = __ldg(static_cast<const uint2*>(a.map) + p);
    return make_float4(bf16_lo(r.x), bf16_hi(r.x), bf16_lo(r.y), bf16_hi(r.y));
  }
}

__device__ __forceinline__ float rec_at(const float4& r, int c) {
  return c == 0 ? r.x : (c == 1 ? r.y : (c == 2 ? r.z : r.w));
}

template <typename TabT>
__device__ __forceinline__ TabT make_tab(double c, double s);
template <>
__device__ __forceinline__ double2 make_tab<double2>(double c, double s) {
  return make_double2(c, s);
}
template <>
__device__ __forceinline__ float2 make_tab<float2>(double c, double s) {
  return make_float2((float)c, (float)s);
}

// Per-thread accumulators: float64 (parity path) or float32 with Kahan
// compensation (precision form).
struct Acc64 {
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  __device__ __forceinline__ void add(int c, double x) { v[c] += x; }
  __device__ __forceinline__ double total(int c) const { return v[c]; }
};
struct AccKahan {
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  float e[4] = {0.f, 0.f, 0.f, 0.f};  // running compensation (minus the lost low bits)
  __device__ __forceinline__ void add(int c, float x) {
    const float y = x - e[c];
    const float t = s[c] + y;
    e[c] = (t - s[c]) - y;
    s[c] = t;
  }
  __device__ __forceinline__ double total(int c) const { return (double)s[c] - (double)e[c]; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Ring table (global memory, built once per nside and footprint reach) and
// the per-sample spin-2 table (shared memory).
// ---------------------------------------------------------------------------

// One RING ring.  Record 0 is a header: z = nside, ta = reach [rad].  The
// fields come in 16-byte pairs in the order the stencil reads them: {z, sth},
// {phi0, dphi}, {ta, inv_dta}, {first32, n, inv_dphi}.
struct __align__(16) RingRec {
  double z;         // ring centre z
  double sth;       // sqrt(max(0, 1 - z^2))
  double phi0;      // longitude of the first pixel
  double dphi;      // pixel spacing
  double ta;        // acos(z)
  double inv_dta;   // 1 / (ta(ir + 1) - ta), correctly rounded (0 for the last ring)
  int first32;      // first pixel index in 32 bits (exact while 12 nside^2 < 2^31)
  int n;            // pixels in the ring
  double inv_dphi;  // 1 / dphi, correctly rounded
  long long first;  // first pixel index
  int cap;          // spin-2 table slots reserved for this ring
  int unused;
};
static_assert(sizeof(RingRec) == 80, "RingRec must be 80 bytes");
static_assert(offsetof(RingRec, phi0) == 16 && offsetof(RingRec, ta) == 32 && offsetof(RingRec, first32) == 48,
              "RingRec pairs must sit on 16-byte boundaries");

// Ring provider backed by the global ring table.
struct TableRings {
  const RingRec* t;
  __device__ __forceinline__ RingData operator()(long long ir) const {
    const RingRec* r = t + ir;
    RingData d;
    d.z = __ldg(&r->z);
    d.ta = __ldg(&r->ta);
    d.phi0 = __ldg(&r->phi0);
    d.dphi = __ldg(&r->dphi);
    d.first = __ldg(&r->first);
    d.n = __ldg(&r->n);
    return d;
  }
  __device__ __forceinline__ double sth(long long ir, const RingData&) const { return __ldg(&t[ir].sth); }
};

// Per-sample spin-2 table: window ring r (ring ir_lo + r) has ring[r] =
// {off, iplo, cap, 0}: slots [off, off + cap) hold cos 2d / sin 2d of its
// in-ring pixels iplo, iplo + 1, ... (mod n).  hdr = {ir_lo in 32 bits, window
// rings (0: no table for this sample), filled slots, 0}.
// A launch reserves ring[0 .. KArgs::ring_cap) (at least 1: ring_win reads
// ring[0] for a sample without a window; at most kRingCap); the table's slots
// follow at spin2_header_bytes(ring_cap).
struct Spin2Tab {
  int4 hdr;
  long long ir_lo;
  long long unused;
  int4 ring[kRingCap];
};
static_assert(offsetof(Spin2Tab, ring) == 32 && sizeof(int4) == 16, "Spin2Tab layout");
__host__ __device__ constexpr size_t spin2_header_bytes(int ring_cap) { return 32 + 16 * (size_t)ring_cap; }

struct Bore {
  double z, sth, phi;
};

// One sample's rotation and boresight in shared memory, written by one thread
// and read by all: the roll about the boresight p (cos/sin psi and 1 - cos
// psi), the recentring about axis k (float64 form with 1 - cos a; for float32
// parameters the reference's float32 inputs, and 1 - (double) cos a), and the
// boresight (z, sin theta, phi) of the spin-2 angle.  Pairs sit on 16-byte
// boundaries for 16-byte shared loads.
struct __align__(16) SampleBlock {
  double px, py, pz, cp, sp, omp;
  double kx, ky, kz, ca, sa, oma;
  float fkx, fky, fkz, fca, fsa, fpad0, fpad1, fpad2;
  double bz, bsth, bphi, bpad;
};
static_assert(sizeof(SampleBlock) == 160, "SampleBlock layout");

// A sample's pointing fields in shared memory, brought there by cp.async one
// sample ahead (field i at byte 4 i for the reference float32 parameters, at
// byte 8 i otherwise).
struct __align__(16) RawFields {
  unsigned long long v[12];
};

template <int PM>
struct SharedFields {
  const KArgs& a;
  const RawFields& raw;
  __device__ __forceinline__ auto operator()(int i) const {
    if constexpr (PM == kParamsRef32)
      return reinterpret_cast<const float*>(raw.v)[i];
    else if constexpr (PM == kAngles)
      return a.angles_f32 ? (double)reinterpret_cast<const float*>(raw.v)[2 * i]
                          : reinterpret_cast<const double*>(raw.v)[i];
    else
      return reinterpret_cast<const double*>(raw.v)[i];
  }
};

// Lane `lane` of one warp starts the copy of field `lane` of sample b into raw
// (cp.async, this GPU's memory); every lane commits its group.
template <int PM>
__device__ __forceinline__ void prefetch_fields(const KArgs& a, long long b, RawFields& raw, int lane) {
  if (lane < field_count<PM>()) {
    const void* src = field_ptr<PM>(a, b, lane);
    if (src != nullptr) {
      const unsigned dst =
          (unsigned)__cvta_generic_to_shared(reinterpret_cast<unsigned char*>(raw.v) + (PM == kParamsRef32 ? 4 : 8) * lane);
      if (field_bytes<PM>(a) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// One thread fills a sample's block from its fields (got: GlobalFields or
// SharedFields); out of line, so that its registers stay out of the pixel loop.
template <int PM, class Get>
__device__ __noinline__ void write_block(const KArgs& a, Get got, bool has_qu, SampleBlock& sb) {
  const SampleRot r = rot_from_fields<PM>(a, got);
  sb.px = r.px;
  sb.py = r.py;
  sb.pz = r.pz;
  sb.cp = r.cp;
  sb.sp = r.sp;
  sb.omp = 1.0 - r.cp;
  sb.kx = r.kx;
  sb.ky = r.ky;
  sb.kz = r.kz;
  sb.ca = r.ca;
  sb.sa = r.sa;
  if constexpr (PM == kParamsRef32) {
    sb.fkx = r.fkx;
    sb.fky = r.fky;
    sb.fkz = r.fkz;
    sb.fca = r.fca;
    sb.fsa = r.fsa;
    sb.oma = 1.0 - (double)r.fca;
  } else {
    sb.oma = 1.0 - r.ca;
  }
  if (has_qu) {
    double z, sth, phi;
    boresight_from_fields<PM>(a, r, got, z, sth, phi);
    sb.bz = z;
    sb.bsth = sth;
    sb.bphi = phi;
  }
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Shared-memory loads that stay inside the pixel loop (the values are the
// same for every pixel of a sample; loading them per pixel keeps them out of
// the registers the evaluation needs).
__device__ __forceinline__ double2 lds_d2(const void* p) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(smem_u32(p)));
  return v;
}
__device__ __forceinline__ double lds_d1(const void* p) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(smem_u32(p)));
  return v;
}
__device__ __forceinline__ float4 lds_f4(const void* p) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"(smem_u32(p)));
  return v;
}
__device__ __forceinline__ int4 lds_i4(const void* p) {
  int4 v;
  asm volatile("ld.shared.v4.s32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(smem_u32(p)));
  return v;
}

__device__ __forceinline__ Bore block_bore(const SampleBlock* sb) {
  const double2 zs = lds_d2(&sb->bz);
  return Bore{zs.x, zs.y, lds_d1(&sb->bphi)};
}

// Rotated beam pixel with the sample's block: the operations of rot_ref32
// (float32 parameters, float32 beam vector) or rot_f64 (float64), with 1 - cos a
// and 1 - cos psi taken from the block (the same values).
__device__ __forceinline__ void rotate_block(const SampleBlock* sb, float vx, float vy, float vz, double& ox,
                                             double& oy, double& oz) {
  const float4 fk = lds_f4(&sb->fkx);  // fkx, fky, fkz, fca
  const float fsa = lds_f4(&sb->fsa).x;
  const double oma = lds_d2(&sb->sa).y;
  const float dkv = fk.x * vx + fk.y * vy + fk.z * vz;
  const float ax = vx * fk.w + (fk.y * vz - fk.z * vy) * fsa;
  const float ay = vy * fk.w + (fk.z * vx - fk.x * vz) * fsa;
  const float az = vz * fk.w + (fk.x * vy - fk.y * vx) * fsa;
  const double rx = (double)ax + (double)(fk.x * dkv) * oma;
  const double ry = (double)ay + (double)(fk.y * dkv) * oma;
  const double rz = (double)az + (double)(fk.z * dkv) * oma;
  const double2 pxy = lds_d2(&sb->px), pzc = lds_d2(&sb->pz), so = lds_d2(&sb->sp);
  const double dpr = pxy.x * rx + pxy.y * ry + pzc.x * rz;
  ox = rx * pzc.y + (pxy.y * rz - pzc.x * ry) * so.x + pxy.x * dpr * so.y;
  oy = ry * pzc.y + (pzc.x * rx - pxy.x * rz) * so.x + pxy.y * dpr * so.y;
  oz = rz * pzc.y + (pxy.x * ry - pxy.y * rx) * so.x + pzc.x * dpr * so.y;
}
__device__ __forceinline__ void rotate_block(const SampleBlock* sb, double vx, double vy, double vz, double& ox,
                                             double& oy, double& oz) {
  const double2 kxy = lds_d2(&sb->kx), kzc = lds_d2(&sb->kz), sao = lds_d2(&sb->sa);
  const double dkv = kxy.x * vx + kxy.y * vy + kzc.x * vz;
  const double rx = vx * kzc.y + (kxy.y * vz - kzc.x * vy) * sao.x + kxy.x * dkv * sao.y;
  const double ry = vy * kzc.y + (kzc.x * vx - kxy.x * vz) * sao.x + kxy.y * dkv * sao.y;
  const double rz = vz * kzc.y + (kxy.x * vy - kxy.y * vx) * sao.x + kzc.x * dkv * sao.y;
  const double2 pxy = lds_d2(&sb->px), pzc = lds_d2(&sb->pz), so = lds_d2(&sb->sp);
  const double dpr = pxy.x * rx + pxy.y * ry + pzc.x * rz;
  ox = rx * pzc.y + (pxy.y * rz - pzc.x * ry) * so.x + pxy.x * dpr * so.y;
  oy = ry * pzc.y + (pzc.x * rx - pxy.x * rz) * so.x + pxy.y * dpr * so.y;
  oz = rz * pzc.y + (pxy.x * ry - pxy.y * rx) * so.x + pzc.x * dpr * so.y;
}

// The float64 form of the block's rotation applied to a float64 vector (the
// footprint centre; the operations of rot_f64).
__device__ __forceinline__ void rotate_block_f64(const SampleBlock& sb, double vx, double vy, double vz, double& ox,
                                                 double& oy, double& oz) {
  const double dkv = sb.kx * vx + sb.ky * vy + sb.kz * vz;
  const double rx = vx * sb.ca + (sb.ky * vz - sb.kz * vy) * sb.sa + sb.kx * dkv * sb.oma;
  const double ry = vy * sb.ca + (sb.kz * vx - sb.kx * vz) * sb.sa + sb.ky * dkv * sb.oma;
  const double rz = vz * sb.ca + (sb.kx * vy - sb.ky * vx) * sb.sa + sb.kz * dkv * sb.oma;
  const double dpr = sb.px * rx + sb.py * ry + sb.pz * rz;
  ox = rx * sb.cp + (sb.py * rz - sb.pz * ry) * sb.sp + sb.px * dpr * sb.omp;
  oy = ry * sb.cp + (sb.pz * rx - sb.px * rz) * sb.sp + sb.py * dpr * sb.omp;
  oz = rz * sb.cp + (sb.px * ry - sb.py * rx) * sb.sp + sb.pz * dpr * sb.omp;
}

template <typename TabT>
__device__ __forceinline__ void spin2_lookup(const Spin2Tab& w, const TabT* tab, long long ring, long long ip,
                                             long long n, double zn, double phin, const Bore& bo, double& c2d,
                                             double& s2d) {
  // ip is the pixel's in-ring index and n its ring's length; the spill case
  // (ip == n) and anything outside the window use direct evaluation.
  const long long r = ring - w.ir_lo;
  if ((unsigned long long)r < (unsigned long long)w.hdr.y && (unsigned long long)ip < (unsigned long long)n) {
    const int4 wr = w.ring[r];
    long long j = ip - wr.y;
    if (j < 0) j += n;
    if (j >= 0 && j < wr.z) {
      const TabT v = tab[wr.x + j];
      c2d = (double)v.x;
      s2d = (double)v.y;
      return;
    }
  }
  const double sth_n = sqrt(max0(1.0 - zn * zn));
  spin2_c2s2(zn, sth_n, phin, bo.z, bo.sth, bo.phi, c2d, s2d);
}

// Beam centre direction (normalised mean of the beam vectors) and the
// largest angle between it and any beam vector; block-wide, once per CTA.
template <int PM, int NT>
__device__ void beam_extent(const KArgs& a, double* s_red, double& cx, double& cy, double& cz, double& radius) {
  constexpr int NW = NT / 32;
  double sx = 0.0, sy = 0.0, sz = 0.0;
  for (long long s = threadIdx.x; s < a.S; s += NT) {
    if constexpr (PM != kParamsRef32) {
      const double* v = static_cast<const double*>(a.vec) + 3 * s;
      sx += v[0];
      sy += v[1];
      sz += v[2];
    } else {
      const float* v = static_cast<const float*>(a.vec) + 3 * s;
      sx += (double)v[0];
      sy += (double)v[1];
      sz += (double)v[2];
    }
  }
  sx = warp_sum(sx);
  sy = warp_sum(sy);
  sz = warp_sum(sz);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    s_red[warp * 4 + 0] = sx;
    s_red[warp * 4 + 1] = sy;
    s_red[warp * 4 + 2] = sz;
  }
  __syncthreads();
  sx = sy = sz = 0.0;
  for (int i = 0; i < NW; ++i) {
    sx += s_red[i * 4 + 0];
    sy += s_red[i * 4 + 1];
    sz += s_red[i * 4 + 2];
  }
  const double nrm = sqrt(sx * sx + sy * sy + sz * sz);
  if (nrm > 0.0) {
    cx = sx / nrm;
    cy = sy / nrm;
    cz = sz / nrm;
  } else {
    cx = 0.0;
    cy = 0.0;
    cz = 1.0;
  }
  double mind = 1.0;
  for (long long s = threadIdx.x; s < a.S; s += NT) {
    double vx, vy, vz;
    if constexpr (PM != kParamsRef32) {
      const double* v = static_cast<const double*>(a.vec) + 3 * s;
      vx = v[0];
      vy = v[1];
      vz = v[2];
    } else {
      const float* v = static_cast<const float*>(a.vec) + 3 * s;
      vx = v[0];
      vy = v[1];
      vz = v[2];
    }
    const double vn = sqrt(vx * vx + vy * vy + vz * vz);
    const double d = vn > 0.0 ? (vx * cx + vy * cy + vz * cz) / vn : -1.0;
    mind = fmin(mind, d);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mind = fmin(mind, __shfl_xor_sync(0xffffffffu, mind, o));
  __syncthreads();
  if (lane == 0) s_red[warp] = mind;
  __syncthreads();
  mind = 1.0;
  for (int i = 0; i < NW; ++i) mind = fmin(mind, s_red[i]);
  __syncthreads();
  radius = acos(clamp1(mind));
}

// ---------------------------------------------------------------------------
// The beam in shared memory.  When the launch leaves room after the spin-2
// table, each CTA copies its job's beam (pixel vectors and weights, in the
// caller's layout) there once with bulk copies (cp.async.bulk, 1-D, this
// GPU's memory, no multicast) on an mbarrier, the unaligned ends of the two
// arrays with plain loads, and the pixel loop reads it from shared memory.
// Every wait is bounded: a wait that runs out is counted in
// g_gather_wait_timeouts (and in the call's error counter), the CTA copies the
// beam with plain loads instead and waits, again bounded, for the bulk copies
// it started before going on.
// ---------------------------------------------------------------------------

constexpr int kStageWaitLimit = 1 << 20;
__device__ unsigned long long g_gather_wait_timeouts;

// Shared-memory bytes of a staged beam of S pixels with vector elements of
// vec_elem bytes: each array rounded up to 16 bytes, plus 16 for the offset
// that keeps a shared copy congruent to its global source modulo 16.
__host__ __device__ constexpr size_t beam_stage_bytes(long long S, size_t vec_elem) {
  return (((size_t)(3 * S) * vec_elem + 15) / 16) * 16 + 16 + (((size_t)S * 4 + 15) / 16) * 16 + 16;
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned done;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(bar), "r"(parity)
               : "memory");
  return done != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  for (int it = 0; it < kStageWaitLimit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// One array of `count` elements of T at global `src` into shared memory at
// `region` (16-byte aligned); returns the shared copy's element 0.  Thread 0
// issues the bulk copy of the 16-byte aligned middle (its bytes are added to
// `tx`); every thread copies its share of the ends.
template <typename T, int NT>
__device__ __forceinline__ T* stage_array(const T* src, long long count, unsigned char* region, unsigned bar,
                                          unsigned& tx, bool issue) {
  const unsigned long long g = reinterpret_cast<unsigned long long>(src);
  const unsigned long long g_end = g + (unsigned long long)count * sizeof(T);
  const unsigned pad = (unsigned)(g & 15u);
  T* dst = reinterpret_cast<T*>(region + pad);
  const unsigned long long body = (g + 15u) & ~15ull, body_end = g_end & ~15ull;
  // elements [0, head) and [tail0, count) go by plain loads (whole elements:
  // the source is element-aligned), [head, tail0) by the bulk copy
  long long head = count, tail0 = count;
  unsigned bytes = 0;
  if (body_end > body) {
    bytes = (unsigned)(body_end - body);
    head = (long long)((body - g) / sizeof(T));
    tail0 = (long long)((body_end - g) / sizeof(T));
  }
  if (bytes > 0 && issue && threadIdx.x == 0) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(region + pad + (body - g))),
                 "l"(body), "r"(bytes), "r"(bar)
                 : "memory");
  }
  tx += bytes;
  const long long ends = head + (count - tail0);
  for (long long e = threadIdx.x; e < (issue ? ends : count); e += NT) {
    const long long i = issue ? (e < head ? e : tail0 + (e - head)) : e;
    dst[i] = src[i];
  }
  return dst;
}

template <typename VecT, int NT>
__device__ void stage_beam(const KArgs& a, unsigned char* region, unsigned long long* bar_mem, const VecT*& vsrc,
                           const float*& bsrc) {
  // (vsrc, bsrc: the shared copies on return)
  const unsigned bar = smem_u32(bar_mem);
  const long long S = a.S;
  unsigned char* vreg = region;
  unsigned char* breg = region + ((3 * S * sizeof(VecT) + 15) / 16) * 16 + 16;
  __syncthreads();  // earlier users of the region (the previous job) are done
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // order this CTA's earlier generic-proxy accesses of the region before the
    // bulk copies' writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  // bytes the bulk copies will deliver (the same in every thread)
  unsigned tx = 0;
  {
    const unsigned long long gv = reinterpret_cast<unsigned long long>(a.vec);
    const unsigned long long gb = reinterpret_cast<unsigned long long>(a.beam);
    const unsigned long long ve = gv + (unsigned long long)(3 * S) * sizeof(VecT), be = gb + (unsigned long long)S * 4;
    const unsigned long long vb = (gv + 15) & ~15ull, vbe = ve & ~15ull, bb = (gb + 15) & ~15ull, bbe = be & ~15ull;
    tx = (unsigned)((vbe > vb ? vbe - vb : 0) + (bbe > bb ? bbe - bb : 0));
  }
  if (threadIdx.x == 0 && tx > 0)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx) : "memory");
  unsigned tx_issued = 0;
  VecT* sv = stage_array<VecT, NT>(static_cast<const VecT*>(a.vec), 3 * S, vreg, bar, tx_issued, true);
  float* sbv = stage_array<float, NT>(a.beam, S, breg, bar, tx_issued, true);
  bool ok = true;
  if (tx > 0) ok = mbar_wait_bounded(bar, 0);
  if (!ok) {
    // the bulk copies did not report back in time: copy everything with plain
    // loads (the same bytes), then give the copies in flight a last bounded wait
    if (threadIdx.x == 0) {
      atomicAdd(&g_gather_wait_timeouts, 1ull);
      if (a.err != nullptr) atomicAdd(a.err, 1ull);
    }
    unsigned dummy = 0;
    stage_array<VecT, NT>(static_cast<const VecT*>(a.vec), 3 * S, vreg, bar, dummy, false);
    stage_array<float, NT>(a.beam, S, breg, bar, dummy, false);
    mbar_wait_bounded(bar, 0);
  }
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
  vsrc = sv;
  bsrc = sbv;
}

// One beam pixel's contribution per component: generic path (64-bit indices,
// any ring provider, any component layout), used without a ring table and for
// non-finite rotated vectors.  err = 1: a stencil pixel fell outside the map,
// nothing to add.
struct Contrib {
  double v[4];
  int err;
};

template <int MODE, bool HAS_QU, typename MapT, class Rings, typename TabT>
__device__ __forceinline__ Contrib generic_terms(const KArgs& a, const SampleBlock* sb, const Rings& rings,
                                                 const Spin2Tab& w, const TabT* tab, double vx, double vy, double vz,
                                                 double phi_w, float bvf) {
  Contrib out{{0.0, 0.0, 0.0, 0.0}, 0};
  const double bv = (double)bvf;
  const Bore bo{sb->bz, sb->bsth, sb->bphi};
  if constexpr (MODE == TODGPU_BILINEAR) {
    const double z = clamp1(vz);
    // Per-neighbour terms are summed in the reference's order k = 0..3.
    double tq = 0.0, tu = 0.0, to[4] = {0.0, 0.0, 0.0, 0.0};
    bool ok = true;
    hp_stencil(a.nside, z, phi_w, rings,
               [&](int k, long long p, double wk, long long ring, long long ip, long long n, double zn,
                   double phin) {
                 if ((unsigned long long)p >= (unsigned long long)a.npix) {
                   ok = false;
                   return;
                 }
                 if constexpr (HAS_QU) {
                   double c2, s2;
                   spin2_lookup(w, tab, ring, ip, n, zn, phin, bo, c2, s2);
                   const double q = map_at<MapT>(a, a.c_q, p);
                   const double u = map_at<MapT>(a, a.c_u, p);
                   const double vq = wk * fma(q, c2, u * s2);
                   const double vu = wk * fma(u, c2, -q * s2);
                   tq = (k == 0) ? vq : tq + vq;
                   tu = (k == 0) ? vu : tu + vu;
                 }
                 for (int c = 0; c < a.C; ++c) {
                   if (HAS_QU && (c == a.c_q || c == a.c_u)) continue;
                   const double m = map_at<MapT>(a, c, p);
                   to[c] = (k == 0) ? wk * m : fma(wk, m, to[c]);
                 }
               });
    if (!ok) {
      out.err = 1;
      return out;
    }
    for (int c = 0; c < a.C; ++c) {
      if (HAS_QU && c == a.c_q)
        out.v[c] = tq * bv;
      else if (HAS_QU && c == a.c_u)
        out.v[c] = tu * bv;
      else
        out.v[c] = to[c] * bv;
    }
  } else {
    const double sin_th = sqrt(max0(vx * vx + vy * vy));
    const Nearest nb = hp_nearest(a.nside, vz, sin_th, phi_w, rings);
    if ((unsigned long long)nb.pix >= (unsigned long long)a.npix) {
      out.err = 1;
      return out;
    }
    if constexpr (HAS_QU) {
      double c2d, s2d;
      spin2_lookup(w, tab, nb.ring, nb.ip, nb.n, nb.zc, nb.phic, bo, c2d, s2d);
      const double qv = map_at<MapT>(a, a.c_q, nb.pix);
      const double uv = map_at<MapT>(a, a.c_u, nb.pix);
      for (int c = 0; c < a.C; ++c) {
        if (c == a.c_q)
          out.v[c] = fma(qv, c2d, uv * s2d) * bv;
        else if (c == a.c_u)
          out.v[c] = fma(uv, c2d, -qv * s2d) * bv;
        else
          out.v[c] = map_x_beam<MapT>(a, c, nb.pix, bvf);
      }
    } else {
      for (int c = 0; c < a.C; ++c) out.v[c] = map_x_beam<MapT>(a, c, nb.pix, bvf);
    }
  }
  return out;
}

// The generic path out of line, in the form that measured faster for each mode:
// bilinear returns its terms by value (adding into the caller's accumulator
// by reference would keep that accumulator in local memory for the whole
// pixel loop: 15 -> 12 local loads per warp-evaluation, +1.3% on config 2);
// nearest adds them itself (by value measured 2.7% slower there).
template <int MODE, bool HAS_QU, typename MapT, class Rings, typename TabT>
__device__ __noinline__ Contrib eval_generic(const KArgs& a, const SampleBlock* sb, const Rings& rings,
                                             const Spin2Tab& w, const TabT* tab, double vx, double vy, double vz,
                                             double phi_w, float bvf) {
  return generic_terms<MODE, HAS_QU, MapT>(a, sb, rings, w, tab, vx, vy, vz, phi_w, bvf);
}

template <int MODE, bool HAS_QU, typename MapT, class Rings, typename TabT, class Acc>
__device__ __noinline__ void eval_generic_into(const KArgs& a, const SampleBlock* sb, const Rings& rings,
                                               const Spin2Tab& w, const TabT* tab, double vx, double vy, double vz,
                                               double phi_w, float bvf, Acc& acc, unsigned long long& nerr) {
  const Contrib r = generic_terms<MODE, HAS_QU, MapT>(a, sb, rings, w, tab, vx, vy, vz, phi_w, bvf);
  if (r.err) {
    ++nerr;
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c < a.C) acc.add(c, r.v[c]);
  }
}

// ---------------------------------------------------------------------------
// Fast path: finite rotated vector, ring table present, nside <= 8192 (all
// ring and pixel indices fit 32 bits).  Same decisions and the same floating
// point operations as the generic path, with 32-bit index arithmetic, ring
// data from the table in 16-byte loads, a compile-time component layout and
// the spin-2 window looked up once per ring.
// ---------------------------------------------------------------------------

constexpr int kLayoutGeneric = 0;  // runtime C, c_q, c_u
constexpr int kLayoutIQU = 1;      // C = 3, Q at 1, U at 2

struct RingFast {
  int n, first;
  double phi0, dphi, z, ta, inv_dphi, inv_dta;
};

__device__ __forceinline__ RingFast ring_fast(const RingRec* rt, int ir) {
  const RingRec* r = rt + ir;
  const double2 zs = __ldg(reinterpret_cast<const double2*>(&r->z));
  const double2 pd = __ldg(reinterpret_cast<const double2*>(&r->phi0));
  const double2 ti = __ldg(reinterpret_cast<const double2*>(&r->ta));
  const int4 fn = __ldg(reinterpret_cast<const int4*>(&r->first32));
  RingFast d;
  d.z = zs.x;
  d.phi0 = pd.x;
  d.dphi = pd.y;
  d.ta = ti.x;
  d.inv_dta = ti.y;
  d.first = fn.x;
  d.n = fn.y;
  d.inv_dphi = __longlong_as_double(((long long)(unsigned)fn.w << 32) | (unsigned)fn.z);
  return d;
}

// The ring above also needs sin theta of its centre.
__device__ __forceinline__ RingFast ring_fast_sth(const RingRec* rt, int ir, double& sth) {
  const RingRec* r = rt + ir;
  const double2 zs = __ldg(reinterpret_cast<const double2*>(&r->z));
  const double2 pd = __ldg(reinterpret_cast<const double2*>(&r->phi0));
  const double2 ti = __ldg(reinterpret_cast<const double2*>(&r->ta));
  const int4 fn = __ldg(reinterpret_cast<const int4*>(&r->first32));
  RingFast d;
  d.z = zs.x;
  sth = zs.y;
  d.phi0 = pd.x;
  d.dphi = pd.y;
  d.ta = ti.x;
  d.inv_dta = ti.y;
  d.first = fn.x;
  d.n = fn.y;
  d.inv_dphi = __longlong_as_double(((long long)(unsigned)fn.w << 32) | (unsigned)fn.z);
  return d;
}

// hp_ring_above for a finite |z| <= 1 (int() of an in-range value truncates).
__device__ __forceinline__ int ring_above_fast(int nside, double z) {
  const double az = fabs(z);
  if (az > kTwoThirds) {
    const int ir = (int)((double)nside * sqrt(3.0 * (1.0 - az)));
    return (z < 0.0) ? 4 * nside - ir - 1 : ir;
  }
  return (int)((double)nside * (2.0 - 1.5 * z));
}

// (x + d) mod n for 0 <= x <= n, 1 <= d <= 2 and n >= 4.
__device__ __forceinline__ int wrap_up(int x, int d, int n) {
  const int v = x + d;
  return v >= n ? v - n : v;
}

// cos(d) for |d| <= kCosSmallMax by its Taylor series through d^6 (the first
// term left out, d^8 / 8!, is below 7e-19 there), in Horner form in d^2.
constexpr double kCosSmallMax = 0.02;
__device__ __forceinline__ double cos_small(double d) {
  const double u = d * d;
  return fma(u, fma(u, fma(u, -1.0 / 720.0, 1.0 / 24.0), -0.5), 1.0);
}

// x / d correctly rounded, from y = 1 / d correctly rounded: the quotient
// x y and two residual corrections by Markstein's theorem (P. Markstein, IBM
// J. Res. Dev. 34(1), 1990: with y within half an ulp of 1/d and q within
// one ulp of x/d, the residual r = x - q d is exact under fma and
// fma(r, y, q) is x/d rounded to nearest).  The first correction brings x y
// (within two ulps) within one ulp, the second rounds correctly.  For finite
// x and d whose quotient and residuals stay in the normal range -- the ring,
// weight and longitude quotients here (|x| < 1e6, 1e-5 < |d| < 7).
__device__ __forceinline__ double div_rn(double x, double d, double y) {
  const double q0 = x * y;
  const double q1 = fma(fma(-q0, d, x), y, q0);
  return fma(fma(-q1, d, x), y, q1);
}
constexpr double kInvTwoPi = 1.0 / kTwoPi;

// Spin-2 window entry of one ring of the sample: {off, iplo, cap} and
// whether the ring lies in the window.
struct RingWin {
  int off, iplo, cap;
  bool in;
};

__device__ __forceinline__ int2 lds_i2(const void* p) {
  int2 v;
  asm volatile("ld.shared.v2.s32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(smem_u32(p)));
  return v;
}

__device__ __forceinline__ RingWin ring_win(const Spin2Tab& w, const int2& hdr, int ring) {
  const unsigned r = (unsigned)(ring - hdr.x);
  RingWin rw;
  rw.in = r < (unsigned)hdr.y;
  const int4 v = lds_i4(&w.ring[rw.in ? r : 0u]);
  rw.off = v.x;
  rw.iplo = v.y;
  rw.cap = v.z;
  return rw;
}

// cos 2d / sin 2d of in-ring pixel ip (of n) from the table, or directly
// (pixel outside the window, spill case ip == n).
template <typename TabT>
__device__ __forceinline__ void spin2_win(const RingWin& rw, const TabT* tab, const SampleBlock* sb, int ip, int n,
                                          double zn, double phin, double& c2d, double& s2d) {
  int j = ip - rw.iplo;
  j += (j >> 31) & n;
  if (rw.in && (unsigned)ip < (unsigned)n && (unsigned)j < (unsigned)rw.cap) {
    const TabT v = tab[rw.off + j];
    c2d = (double)v.x;
    s2d = (double)v.y;
    return;
  }
  const Bore bo = block_bore(sb);
  const double sth_n = sqrt(max0(1.0 - zn * zn));
  spin2_c2s2(zn, sth_n, phin, bo.z, bo.sth, bo.phi, c2d, s2d);
}

// The bilinear stencil of hp_stencil with 32-bit indices; tw is in [0, n]
// for finite phi in [0, 2 pi], so int(tw) is a plain truncation.  visit(k,
// pixel, weight, in-ring index, ring length, ring z, pixel phi, ring window).
template <bool HAS_QU, class Visit>
__device__ __forceinline__ void stencil_fast(int nside, double z, double phi_w, const RingRec* rt, const Spin2Tab& w,
                                             const int2& hdr, Visit&& visit) {
  const int ir_above = ring_above_fast(nside, z);
  RingWin ra_w{0, 0, 0, false};
  if (ir_above == 0) {
    const RingFast ra = ring_fast(rt, 1);
    if constexpr (HAS_QU) ra_w = ring_win(w, hdr, 1);
    const double tw = py_fmod_pos((phi_w - ra.phi0) / ra.dphi, (double)ra.n);
    const int ip = (int)tw;
    const double frac = tw - (double)ip;
    const int ip2 = wrap_up(ip, 1, ra.n);
    const int o1 = wrap_up(ip, 2, ra.n), o2 = wrap_up(ip2, 2, ra.n);
    const double theta = acos(z);
    const double wt = theta / ra.ta;
    const double nf = (1.0 - wt) * 0.25;
    visit(0, ra.first + o1, nf, o1, ra.n, ra.z, ra.phi0 + (double)o1 * ra.dphi, ra_w);
    visit(1, ra.first + o2, nf, o2, ra.n, ra.z, ra.phi0 + (double)o2 * ra.dphi, ra_w);
    visit(2, ra.first + ip, (1.0 - frac) * wt + nf, ip, ra.n, ra.z, ra.phi0 + (double)ip * ra.dphi, ra_w);
    visit(3, ra.first + ip2, frac * wt + nf, ip2, ra.n, ra.z, ra.phi0 + (double)ip2 * ra.dphi, ra_w);
  } else if (ir_above == 4 * nside - 1) {
    const int ir_last = 4 * nside - 1;
    const RingFast ra = ring_fast(rt, ir_last);
    if constexpr (HAS_QU) ra_w = ring_win(w, hdr, ir_last);
    const double tw = py_fmod_pos((phi_w - ra.phi0) / ra.dphi, (double)ra.n);
    const int ip = (int)tw;
    const double frac = tw - (double)ip;
    const int ip2 = wrap_up(ip, 1, ra.n);
    const int o1 = wrap_up(ip, 2, ra.n), o2 = wrap_up(ip2, 2, ra.n);
    const double theta = acos(z);
    const double ws = (theta - ra.ta) / (kPi - ra.ta);
    const double sf = ws * 0.25;
    visit(0, ra.first + ip, (1.0 - frac) * (1.0 - ws) + sf, ip, ra.n, ra.z, ra.phi0 + (double)ip * ra.dphi, ra_w);
    visit(1, ra.first + ip2, frac * (1.0 - ws) + sf, ip2, ra.n, ra.z, ra.phi0 + (double)ip2 * ra.dphi, ra_w);
    visit(2, ra.first + o1, sf, o1, ra.n, ra.z, ra.phi0 + (double)o1 * ra.dphi, ra_w);
    visit(3, ra.first + o2, sf, o2, ra.n, ra.z, ra.phi0 + (double)o2 * ra.dphi, ra_w);
  } else {
    const int ir_below = ir_above + 1;
    double sth_a;
    const RingFast ra = ring_fast_sth(rt, ir_above, sth_a);
    // of the ring below only its colatitude is needed before the ring above's
    // neighbours; the rest is loaded after them
    const double ta_b = __ldg(&rt[ir_below].ta);
    double dta;
    if (!dtheta_small(z, ra.z, sth_a, dta)) dta = acos(z) - ra.ta;
    const double wb = div_rn(dta, ta_b - ra.ta, ra.inv_dta);
    const double wa = 1.0 - wb;
    double tw = py_fmod_pos(div_rn(phi_w - ra.phi0, ra.dphi, ra.inv_dphi), (double)ra.n);
    const int ia = (int)tw;
    const double fa = tw - (double)ia;
    const int ia1 = wrap_up(ia, 1, ra.n);
    if constexpr (HAS_QU) ra_w = ring_win(w, hdr, ir_above);
    visit(0, ra.first + ia, wa * (1.0 - fa), ia, ra.n, ra.z, ra.phi0 + (double)ia * ra.dphi, ra_w);
    visit(1, ra.first + ia1, wa * fa, ia1, ra.n, ra.z, ra.phi0 + (double)ia1 * ra.dphi, ra_w);
    const RingFast rb = ring_fast(rt, ir_below);
    tw = py_fmod_pos(div_rn(phi_w - rb.phi0, rb.dphi, rb.inv_dphi), (double)rb.n);
    const int ib = (int)tw;
    const double fb = tw - (double)ib;
    const int ib1 = wrap_up(ib, 1, rb.n);
    RingWin rb_w{0, 0, 0, false};
    if constexpr (HAS_QU) rb_w = ring_win(w, hdr, ir_below);
    visit(2, rb.first + ib, wb * (1.0 - fb), ib, rb.n, rb.z, rb.phi0 + (double)ib * rb.dphi, rb_w);
    visit(3, rb.first + ib1, wb * fb, ib1, rb.n, rb.z, rb.phi0 + (double)ib1 * rb.dphi, rb_w);
  }
}

template <int LAYOUT>
struct Chan {
  int C, q, u;
  __device__ __forceinline__ explicit Chan(const KArgs& a) : C(a.C), q(a.c_q), u(a.c_u) {}
};
template <>
struct Chan<kLayoutIQU> {
  static constexpr int C = 3, q = 1, u = 2;
  __device__ __forceinline__ explicit Chan(const KArgs&) {}
};

template <typename MapT>
__device__ __forceinline__ double map_i(const KArgs& a, int c, int p) {
  if constexpr (std::is_same<MapT, PackF64>::value)
    return __ldg(static_cast<const double*>(a.map) + 4LL * p + c);
  else
    return (double)__ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
}

template <typename MapT>
__device__ __forceinline__ double map_x_beam_i(const KArgs& a, int c, int p, float bv) {
  if constexpr (std::is_same<MapT, PackF64>::value) {
    return __ldg(static_cast<const double*>(a.map) + 4LL * p + c) * (double)bv;
  } else {
    const MapT m = __ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
    if constexpr (sizeof(MapT) == 4)
      return (double)(m * bv);
    else
      return m * (double)bv;
  }
}

// A pixel's map values for the float64 bilinear path: planar maps read each
// component where it is used; PackF64 records are read as two 16-byte loads.
template <typename MapT>
struct PixelVals {
  const KArgs& a;
  int p;
  __device__ __forceinline__ PixelVals(const KArgs& a_, int p_) : a(a_), p(p_) {}
  __device__ __forceinline__ double operator()(int c) const { return map_i<MapT>(a, c, p); }
};
template <>
struct PixelVals<PackF64> {
  double2 lo, hi;
  __device__ __forceinline__ PixelVals(const KArgs& a, int p)
      : lo(__ldg(static_cast<const double2*>(a.map) + 2LL * p)),
        hi(__ldg(static_cast<const double2*>(a.map) + 2LL * p + 1)) {}
  __device__ __forceinline__ double operator()(int c) const {
    return c == 0 ? lo.x : (c == 1 ? lo.y : (c == 2 ? hi.x : hi.y));
  }
};

// The nearest rule's ring data: n, phi0, dphi, z and sin theta of ring ir.
struct RingNear {
  int n, first;
  double phi0, dphi, z, sth;
};
__device__ __forceinline__ RingNear ring_near(const RingRec* rt, int ir) {
  const RingRec* r = rt + ir;
  const double2 zs = __ldg(reinterpret_cast<const double2*>(&r->z));
  const double2 pd = __ldg(reinterpret_cast<const double2*>(&r->phi0));
  const int2 fn = __ldg(reinterpret_cast<const int2*>(&r->first32));
  return RingNear{fn.y, fn.x, pd.x, pd.y, zs.x, zs.y};
}

// Per-neighbour mixing of the bilinear path, in the reference's k = 0..3 order:
// float64 for planar maps and float64 records, float32 for packed records
// (precision form); term(c) is what the pixel adds to component c.
template <typename MapT, int LAYOUT, bool HAS_QU>
struct BilinearMix {
  static constexpr bool kPacked = MapTraits<MapT>::packed;
  using R = typename std::conditional<kPacked, float, double>::type;
  R tq = 0, tu = 0, to[4] = {0, 0, 0, 0};
  __device__ __forceinline__ void visit(const KArgs& a, const Chan<LAYOUT>& ch, int k, int p, double wk, double c2,
                                        double s2) {
    if constexpr (kPacked) {
      const float4 rec = load_rec<MapT>(a, p);
      const float wf = (float)wk;
      if constexpr (HAS_QU) {
        const float c2f = (float)c2, s2f = (float)s2;
        const float q = rec_at(rec, ch.q), u = rec_at(rec, ch.u);
        const float vq = wf * fmaf(q, c2f, u * s2f);
        const float vu = wf * fmaf(u, c2f, -q * s2f);
        tq = (k == 0) ? vq : tq + vq;
        tu = (k == 0) ? vu : tu + vu;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ch.C) break;
        if (HAS_QU && (c == ch.q || c == ch.u)) continue;
        to[c] = (k == 0) ? wf * rec_at(rec, c) : fmaf(wf, rec_at(rec, c), to[c]);
      }
    } else {
      const PixelVals<MapT> pv(a, p);
      if constexpr (HAS_QU) {
        const double q = pv(ch.q);
        const double u = pv(ch.u);
        const double vq = wk * fma(q, c2, u * s2);
        const double vu = wk * fma(u, c2, -q * s2);
        tq = (k == 0) ? vq : tq + vq;
        tu = (k == 0) ? vu : tu + vu;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ch.C) break;
        if (HAS_QU && (c == ch.q || c == ch.u)) continue;
        const double m = pv(c);
        to[c] = (k == 0) ? wk * m : fma(wk, m, to[c]);
      }
    }
  }
  __device__ __forceinline__ double term(const Chan<LAYOUT>& ch, int c, float bvf) const {
    if constexpr (kPacked) {
      return (double)((HAS_QU && c == ch.q) ? tq * bvf : ((HAS_QU && c == ch.u) ? tu * bvf : to[c] * bvf));
    } else {
      const double bv = (double)bvf;
      return (HAS_QU && c == ch.q) ? tq * bv : ((HAS_QU && c == ch.u) ? tu * bv : to[c] * bv);
    }
  }
};

// The bilinear stencil in the common case, without branches per neighbour:
// a query between two rings away from the poles, both longitude quotients
// inside their rings (no modulo, no spill into the next ring) and, with Q and
// U, all four neighbours in the sample's spin-2 table.  The same operations
// on the same values as stencil_fast + spin2_win; returns false (having added
// nothing) when any of these does not hold, for the caller to take the full
// path.
template <bool HAS_QU, typename MapT, int LAYOUT, typename TabT, class Acc>
__device__ __forceinline__ bool bilinear_lean(const KArgs& a, const RingRec* rt, const Spin2Tab& w,
                                              const TabT* tab, const int2& hdr, double z, double phi_w, float bvf,
                                              Acc& acc) {
  const int nside = (int)a.nside;
  const int ir_above = ring_above_fast(nside, z);
  if (ir_above == 0 || ir_above == 4 * nside - 1) return false;
  const int ir_below = ir_above + 1;
  double sth_a;
  const RingFast ra = ring_fast_sth(rt, ir_above, sth_a);
  const RingFast rb = ring_fast(rt, ir_below);
  // longitude quotients: py_fmod_pos without its fmod branch
  const double xa = div_rn(phi_w - ra.phi0, ra.dphi, ra.inv_dphi);
  const double xb = div_rn(phi_w - rb.phi0, rb.dphi, rb.inv_dphi);
  const double na = (double)ra.n, nb = (double)rb.n;
  if (!(fabs(xa) < na && fabs(xb) < nb)) return false;
  const double twa = xa < 0.0 ? xa + na : (xa == 0.0 ? 0.0 : xa);
  const double twb = xb < 0.0 ? xb + nb : (xb == 0.0 ? 0.0 : xb);
  const int ia = (int)twa, ib = (int)twb;
  if (ia >= ra.n || ib >= rb.n) return false;  // the spill into the next ring
  const int ia1 = ia + 1 == ra.n ? 0 : ia + 1, ib1 = ib + 1 == rb.n ? 0 : ib + 1;
  double c2[4] = {1.0, 1.0, 1.0, 1.0}, s2[4] = {0.0, 0.0, 0.0, 0.0};
  if constexpr (HAS_QU) {
    const RingWin wa = ring_win(w, hdr, ir_above), wb = ring_win(w, hdr, ir_below);
    int j0 = ia - wa.iplo, j1 = ia1 - wa.iplo, j2 = ib - wb.iplo, j3 = ib1 - wb.iplo;
    j0 += (j0 >> 31) & ra.n;
    j1 += (j1 >> 31) & ra.n;
    j2 += (j2 >> 31) & rb.n;
    j3 += (j3 >> 31) & rb.n;
    if (!(wa.in && wb.in && (unsigned)j0 < (unsigned)wa.cap && (unsigned)j1 < (unsigned)wa.cap &&
          (unsigned)j2 < (unsigned)wb.cap && (unsigned)j3 < (unsigned)wb.cap))
      return false;
    const TabT t0 = tab[wa.off + j0], t1 = tab[wa.off + j1], t2 = tab[wb.off + j2], t3 = tab[wb.off + j3];
    c2[0] = (double)t0.x;
    s2[0] = (double)t0.y;
    c2[1] = (double)t1.x;
    s2[1] = (double)t1.y;
    c2[2] = (double)t2.x;
    s2[2] = (double)t2.y;
    c2[3] = (double)t3.x;
    s2[3] = (double)t3.y;
  }
  double dta;
  if (!dtheta_small(z, ra.z, sth_a, dta)) dta = acos(z) - ra.ta;
  const double wgt_b = div_rn(dta, rb.ta - ra.ta, ra.inv_dta);
  const double wgt_a = 1.0 - wgt_b;
  const double fa = twa - (double)ia, fb = twb - (double)ib;
  const Chan<LAYOUT> ch(a);
  BilinearMix<MapT, LAYOUT, HAS_QU> mix;
  mix.visit(a, ch, 0, ra.first + ia, wgt_a * (1.0 - fa), c2[0], s2[0]);
  mix.visit(a, ch, 1, ra.first + ia1, wgt_a * fa, c2[1], s2[1]);
  mix.visit(a, ch, 2, rb.first + ib, wgt_b * (1.0 - fb), c2[2], s2[2]);
  mix.visit(a, ch, 3, rb.first + ib1, wgt_b * fb, c2[3], s2[3]);
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (c >= ch.C) break;
    acc.add(c, mix.term(ch, c, bvf));
  }
  return true;
}

// The full bilinear fast path (poles, ring ends, spills, neighbours outside
// the table), out of line, returning its terms by value.
template <bool HAS_QU, typename MapT, int LAYOUT, typename TabT>
__device__ __noinline__ Contrib bilinear_full(const KArgs& a, const SampleBlock* sb, const RingRec* rt,
                                              const Spin2Tab& w, const TabT* tab, int2 hdr, double z, double phi_w,
                                              float bvf) {
  const Chan<LAYOUT> ch(a);
  BilinearMix<MapT, LAYOUT, HAS_QU> mix;
  stencil_fast<HAS_QU>((int)a.nside, z, phi_w, rt, w, hdr,
                       [&](int k, int p, double wk, int ip, int n, double zn, double phin, const RingWin& rw) {
                         double c2 = 1.0, s2 = 0.0;
                         if constexpr (HAS_QU) spin2_win(rw, tab, sb, ip, n, zn, phin, c2, s2);
                         mix.visit(a, ch, k, p, wk, c2, s2);
                       });
  Contrib out{{0.0, 0.0, 0.0, 0.0}, 0};
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    if (c >= ch.C) break;
    out.v[c] = mix.term(ch, c, bvf);
  }
  return out;
}

// The nearest rule's full path (poles and their neighbourhood, candidates
// more than 0.02 rad apart in longitude, near-ties, neighbours outside the
// spin-2 table), out of line, returning its terms by value.
template <bool HAS_QU, typename MapT, int LAYOUT, typename TabT>
__device__ __noinline__ Contrib nearest_full(const KArgs& a, const SampleBlock* sb, const RingRec* rt,
                                             const Spin2Tab& w, const TabT* tab, int2 hdr, double vx, double vy,
                                             double vz, double phi_w, float bvf) {
  constexpr bool kPacked = MapTraits<MapT>::packed;
  const Chan<LAYOUT> ch(a);
  const int nside = (int)a.nside;
  const double bv = (double)bvf;
  Contrib out{{0.0, 0.0, 0.0, 0.0}, 0};
  // nearest: unclamped z; |z| > 1 makes the reference's ring_above NaN-based
  // and the clamp then picks ring 1 (numba_healpy.py:62-70, tod_nearest.py:115-120)
  const double sin_th = sqrt(max0(vx * vx + vy * vy));
  int ir_above;
  if (fabs(vz) <= 1.0) {
    ir_above = ring_above_fast(nside, vz);
    ir_above = ir_above < 1 ? 1 : (ir_above > 4 * nside - 2 ? 4 * nside - 2 : ir_above);
  } else {
    ir_above = 1;
  }
  // The four candidates: two pixels on each of rings ir_above and
  // ir_above + 1, ranked by the cosine of their angular distance.  A first
  // pass evaluates cos(phi_w - phic) by cos_small where the difference is at
  // most kCosSmallMax (cos() beyond); the two differ by < 2e-15, so a lead of more
  // than 1e-13 over the runner-up picks the pixel that ranking by cos()
  // picks.  A closer call is ranked again by cos() itself -- the same
  // expression, order and strict comparison -- so the pixel is always the
  // one of ranking by cos() throughout.
  int best_g = -1, best_ip = 0;
  const RingNear rg0 = ring_near(rt, ir_above), rg1 = ring_near(rt, ir_above + 1);
  {
    double lead = -3.0, runner = -3.0;
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const RingNear& r = g == 0 ? rg0 : rg1;
      int ipb = (int)div_rn(phi_w * (double)r.n, kTwoPi, kInvTwoPi);
      if (ipb >= r.n) ipb -= r.n;
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int ip = (t == 0) ? ipb : wrap_up(ipb, 1, r.n);
        const double dl = phi_w - (r.phi0 + (double)ip * r.dphi);
        const double cosd = sin_th * r.sth * (fabs(dl) <= kCosSmallMax ? cos_small(dl) : cos(dl)) + vz * r.z;
        if (cosd > lead) {
          runner = lead;
          lead = cosd;
          best_g = g;
          best_ip = ip;
        } else if (cosd > runner) {
          runner = cosd;
        }
      }
    }
    if (!(lead - runner > 1e-13)) {
      double best_cos = -2.0;
      best_g = -1;
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        const RingNear& r = g == 0 ? rg0 : rg1;
        int ipb = (int)(phi_w * (double)r.n / kTwoPi);
        if (ipb >= r.n) ipb -= r.n;
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int ip = (t == 0) ? ipb : wrap_up(ipb, 1, r.n);
          const double phic = r.phi0 + (double)ip * r.dphi;
          const double cosd = sin_th * r.sth * cos(phi_w - phic) + vz * r.z;
          if (cosd > best_cos) {
            best_cos = cosd;
            best_g = g;
            best_ip = ip;
          }
        }
      }
    }
  }
  int best_pix = 0, best_n = 1, best_ring = 0;
  double best_zc = 0.0, best_phic = 0.0;
  if (best_g >= 0) {
    const RingNear& r = best_g == 0 ? rg0 : rg1;
    best_ring = ir_above + best_g;
    best_n = r.n;
    best_pix = r.first + best_ip;
    best_zc = r.z;
    best_phic = r.phi0 + (double)best_ip * r.dphi;
  } else {
    best_ip = 0;
  }
  RingWin rw{0, 0, 0, false};
  if constexpr (HAS_QU) rw = ring_win(w, hdr, best_ring);
  if constexpr (kPacked) {
    const float4 rec = load_rec<MapT>(a, best_pix);
    float c2f = 1.f, s2f = 0.f;
    if constexpr (HAS_QU) {
      double c2d, s2d;
      spin2_win(rw, tab, sb, best_ip, best_n, best_zc, best_phic, c2d, s2d);
      c2f = (float)c2d;
      s2f = (float)s2d;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      if (HAS_QU && c == ch.q)
        out.v[c] = (double)(fmaf(rec_at(rec, ch.q), c2f, rec_at(rec, ch.u) * s2f) * bvf);
      else if (HAS_QU && c == ch.u)
        out.v[c] = (double)(fmaf(rec_at(rec, ch.u), c2f, -rec_at(rec, ch.q) * s2f) * bvf);
      else
        out.v[c] = (double)(rec_at(rec, c) * bvf);
    }
  } else if constexpr (HAS_QU) {
    double c2d, s2d;
    spin2_win(rw, tab, sb, best_ip, best_n, best_zc, best_phic, c2d, s2d);
    const double qv = map_i<MapT>(a, ch.q, best_pix);
    const double uv = map_i<MapT>(a, ch.u, best_pix);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      if (c == ch.q)
        out.v[c] = (double)(fma(qv, c2d, uv * s2d) * bv);
      else if (c == ch.u)
        out.v[c] = (double)(fma(uv, c2d, -qv * s2d) * bv);
      else
        out.v[c] = (double)(map_x_beam_i<MapT>(a, c, best_pix, bvf));
    }
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      out.v[c] = (double)(map_x_beam_i<MapT>(a, c, best_pix, bvf));
    }
  }
  return out;
}

// The nearest rule in the common case, without branches: a query within the
// rings of the map (|z| <= 1), all four candidates within kCosSmallMax of it in
// longitude (so ranked by cos_small), a lead over the runner-up above 1e-13
// (so no re-ranking by cos()), and with Q and U the chosen pixel in the
// sample's spin-2 table.  The same operations on the same values as the full
// path; returns false (having added nothing) when any of these does not hold.
template <bool HAS_QU, typename MapT, int LAYOUT, typename TabT, class Acc>
__device__ __forceinline__ bool nearest_lean(const KArgs& a, const RingRec* rt, const Spin2Tab& w, const TabT* tab,
                                             const int2& hdr, double vx, double vy, double vz, double phi_w,
                                             float bvf, Acc& acc) {
  constexpr bool kPacked = MapTraits<MapT>::packed;
  const int nside = (int)a.nside;
  if (!(fabs(vz) <= 1.0)) return false;
  const double sin_th = sqrt(max0(vx * vx + vy * vy));
  int ir_above = ring_above_fast(nside, vz);
  ir_above = ir_above < 1 ? 1 : (ir_above > 4 * nside - 2 ? 4 * nside - 2 : ir_above);
  const RingNear rg0 = ring_near(rt, ir_above), rg1 = ring_near(rt, ir_above + 1);
  int best_g = -1, best_ip = 0;
  double lead = -3.0, runner = -3.0;
  bool small = true;
#pragma unroll
  for (int g = 0; g < 2; ++g) {
    const RingNear& r = g == 0 ? rg0 : rg1;
    int ipb = (int)div_rn(phi_w * (double)r.n, kTwoPi, kInvTwoPi);
    if (ipb >= r.n) ipb -= r.n;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int ip = (t == 0) ? ipb : wrap_up(ipb, 1, r.n);
      const double dl = phi_w - (r.phi0 + (double)ip * r.dphi);
      small = small && fabs(dl) <= kCosSmallMax;
      const double cosd = sin_th * r.sth * cos_small(dl) + vz * r.z;
      if (cosd > lead) {
        runner = lead;
        lead = cosd;
        best_g = g;
        best_ip = ip;
      } else if (cosd > runner) {
        runner = cosd;
      }
    }
  }
  if (!(small && lead - runner > 1e-13 && best_g >= 0)) return false;
  const RingNear& r = best_g == 0 ? rg0 : rg1;
  const int best_pix = r.first + best_ip;
  double c2d = 1.0, s2d = 0.0;
  if constexpr (HAS_QU) {
    const RingWin rw = ring_win(w, hdr, ir_above + best_g);
    int j = best_ip - rw.iplo;
    j += (j >> 31) & r.n;
    if (!(rw.in && (unsigned)j < (unsigned)rw.cap)) return false;
    const TabT v = tab[rw.off + j];
    c2d = (double)v.x;
    s2d = (double)v.y;
  }
  const Chan<LAYOUT> ch(a);
  if constexpr (kPacked) {
    const float4 rec = load_rec<MapT>(a, best_pix);
    const float c2f = (float)c2d, s2f = (float)s2d;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      if (HAS_QU && c == ch.q)
        acc.add(c, fmaf(rec_at(rec, ch.q), c2f, rec_at(rec, ch.u) * s2f) * bvf);
      else if (HAS_QU && c == ch.u)
        acc.add(c, fmaf(rec_at(rec, ch.u), c2f, -rec_at(rec, ch.q) * s2f) * bvf);
      else
        acc.add(c, rec_at(rec, c) * bvf);
    }
  } else if constexpr (HAS_QU) {
    const double bv = (double)bvf;
    const double qv = map_i<MapT>(a, ch.q, best_pix);
    const double uv = map_i<MapT>(a, ch.u, best_pix);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      if (c == ch.q)
        acc.add(c, fma(qv, c2d, uv * s2d) * bv);
      else if (c == ch.u)
        acc.add(c, fma(uv, c2d, -qv * s2d) * bv);
      else
        acc.add(c, map_x_beam_i<MapT>(a, c, best_pix, bvf));
    }
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (c >= ch.C) break;
      acc.add(c, map_x_beam_i<MapT>(a, c, best_pix, bvf));
    }
  }
  return true;
}

// One beam pixel on the fast path: the branch-free common case of its mode,
// else that mode's full path out of line.
template <int MODE, bool HAS_QU, typename MapT, int LAYOUT, typename TabT, class Acc>
__device__ __forceinline__ void eval_fast(const KArgs& a, const SampleBlock* sb, const RingRec* rt,
                                          const Spin2Tab& w, const TabT* tab, double vx, double vy, double vz,
                                          double phi_w, float bvf, Acc& acc) {
  const Chan<LAYOUT> ch(a);
  int2 hdr = make_int2(0, 0);  // {first window ring, window rings}
  if constexpr (HAS_QU) hdr = lds_i2(&w.hdr);
  if constexpr (MODE == TODGPU_BILINEAR) {
    const double z = clamp1(vz);
    if (!bilinear_lean<HAS_QU, MapT, LAYOUT>(a, rt, w, tab, hdr, z, phi_w, bvf, acc)) {
      const Contrib r = bilinear_full<HAS_QU, MapT, LAYOUT>(a, sb, rt, w, tab, hdr, z, phi_w, bvf);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ch.C) break;
        acc.add(c, r.v[c]);
      }
    }
  } else {
    if (!nearest_lean<HAS_QU, MapT, LAYOUT>(a, rt, w, tab, hdr, vx, vy, vz, phi_w, bvf, acc)) {
      const Contrib r = nearest_full<HAS_QU, MapT, LAYOUT>(a, sb, rt, w, tab, hdr, vx, vy, vz, phi_w, bvf);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= ch.C) break;
        acc.add(c, r.v[c]);
      }
    }
  }
}

// Flush the per-warp partial sums of sample `b` into tod (fixed order).
template <int NW>
__device__ __forceinline__ void flush_sample(const KArgs& a, const double* s_red, long long b) {
  for (int c = 0; c < a.C; ++c) {
    double v = 0.0;
    for (int i = 0; i < NW; ++i) v += s_red[i * 4 + c];
    a.tod[(long long)c * a.tod_stride + b] += v;
  }
}

// Footprint window of one sample, by the kSetupThreads setup threads (warps
// 0 and 1) together: the window rings about the footprint centre u, each
// ring's slots and their offsets in the spin-2 table, into w.  Out of line so
// that its registers do not weigh on the evaluation loop around it.
constexpr int kSetupThreads = 64;
static __device__ __noinline__ void footprint_window(const KArgs& a, const RingRec* rt, Spin2Tab& w, double ux,
                                                     double uy, double uz, double reach) {
  const int lane = threadIdx.x & 31;
  const double theta_u = acos(clamp1(uz));
  double phi_u = atan2(uy, ux);
  if (phi_u < 0.0) phi_u += kTwoPi;
  const double th_lo = theta_u - reach, th_hi = theta_u + reach;
  long long ir_lo = th_lo <= 0.0 ? 1 : hp_ring_above(a.nside, cos(th_lo));
  long long ir_hi = th_hi >= kPi ? 4 * a.nside - 1 : hp_ring_above(a.nside, cos(th_hi)) + 1;
  ir_lo = max(ir_lo, 1LL);
  ir_hi = min(ir_hi, 4 * a.nside - 1);
  // a non-finite footprint centre gives an empty or invalid window: no table
  const long long nr = ir_hi - ir_lo + 1;
  bool fits = nr > 0 && nr <= a.ring_cap && ir_lo >= 1 && ir_hi <= 4 * a.nside - 1;
  // Slots per window ring: the ring's stretch of the footprint disc (radius
  // reach about (theta_u, phi_u)), at most what the ring table reserves
  // for any footprint of that reach.  Away from the poles the disc's
  // half-width in longitude on a ring at colatitude theta_r is
  // sqrt(reach^2 - (theta_r - theta_u)^2) / sin theta_r to within a
  // percent for reach < 0.05; 2% margin and the rounding up of the
  // half-width keep every stencil pixel in.  (A pixel outside its ring's
  // slots is still evaluated, directly; only the cost changes.)
  const bool disc = reach < 0.05 && theta_u - reach > 0.1 && theta_u + reach < kPi - 0.1;
  if (fits) {
    for (int t = threadIdx.x; t < nr; t += kSetupThreads) {
      const RingRec* r = rt + ir_lo + t;
      const int n = __ldg(&r->n);
      int cnt = __ldg(&r->cap);
      if (disc) {
        const double dth = __ldg(&r->ta) - theta_u;
        const double h2 = reach * reach - dth * dth;
        const int k = h2 > 0.0 ? (int)ceil(1.02 * sqrt(h2) / __ldg(&r->sth) * __ldg(&r->inv_dphi)) : 0;
        cnt = min(cnt, 2 * k + 1);
      }
      int iplo = 0;
      if (cnt < n) {
        const double c = floor((phi_u - __ldg(&r->phi0)) / __ldg(&r->dphi));
        iplo = (int)py_imod((long long)c - (cnt - 1) / 2, n);
      }
      w.ring[t].y = iplo;
      w.ring[t].z = cnt;
    }
  }
  // slot offsets: exclusive prefix sum of the counts, by warp 0 once both
  // setup warps have written theirs
  asm volatile("bar.sync 1, %0;" ::"n"(kSetupThreads) : "memory");
  if (threadIdx.x < 32) {
    int carry = 0;
    if (fits) {
      for (int b0 = 0; b0 < (int)nr; b0 += 32) {
        const int t = b0 + lane;
        const int own = t < nr ? w.ring[t].z : 0;
        int v = own;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, v, o);
          if (lane >= o) v += y;
        }
        if (t < nr) w.ring[t].x = carry + v - own;
        carry += __shfl_sync(0xffffffffu, v, 31);
      }
    }
    fits = fits && carry <= a.tab_cap;
    if (threadIdx.x == 0) {
      w.ir_lo = ir_lo;
      w.hdr = make_int4((int)ir_lo, fits ? (int)nr : 0, fits ? carry : 0, 0);
    }
  }
}

// Samples of tiles t = t_begin, t_begin + t_step, ... < t_end of one job (one
// beam entry over one batch of samples; tile t holds samples [t tile,
// min(B, (t + 1) tile))), by the whole CTA.  With a ring table:
// ring data come from it and, when the entry carries Q and U, each sample's
// footprint gets a spin-2 table in shared memory.  Without one: everything is
// evaluated directly.  Each sample's rotation and boresight are derived by one
// thread, one sample ahead, into a double-buffered shared block that all
// threads read.  The beam is read from shared memory when the launch staged
// it there (a.beam_stage), else from global memory.  All threads of the CTA
// must call it together.
template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT, int NT>
__device__ void run_samples(const KArgs& a, long long t_begin, long long t_end, long long t_step, long long tile,
                            unsigned char* smem_raw, double* s_red) {
  constexpr int NW = NT / 32;
  static_assert(NT >= 2 * kSetupThreads && kSumLanes % NT == 0, "CTA of 128 or 256 threads");
  Spin2Tab& w = *reinterpret_cast<Spin2Tab*>(smem_raw);
  using TabT = typename MapTraits<MapT>::Tab;
  using Acc = typename std::conditional<MapTraits<MapT>::packed, AccKahan, Acc64>::type;
  using VecT = typename std::conditional<PM == kParamsRef32, float, double>::type;
  // window rings of the table header (a.ring_cap; a constant in the narrow shape)
  const int hdr_rings = NT == kNTNarrow ? kRingCapNarrow : a.ring_cap;
  TabT* tab = reinterpret_cast<TabT*>(smem_raw + spin2_header_bytes(hdr_rings));
  __shared__ SampleBlock s_blk[2];
  __shared__ __align__(8) unsigned long long s_bar;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const RingRec* rt = static_cast<const RingRec*>(a.ring_table);
  const bool fast = rt != nullptr && a.nside <= 8192;
  double cx = 0.0, cy = 0.0, cz = 1.0, reach = 0.0;
  bool use_tab = false;
  if (rt != nullptr && HAS_QU) {
    double rbeam;
    beam_extent<PM, NT>(a, s_red, cx, cy, cz, rbeam);
    // every stencil neighbour centre lies within 1.7/nside rad of the query
    // (one ring spacing plus one pixel width; the opposite pair around a pole
    // within twice the colatitude of ring 1); 2/nside leaves margin, plus
    // slack for the float32 parameter rounding.  A neighbour outside the
    // window is still evaluated correctly (directly), only slower (measured:
    // 3/nside and 5% more slots per ring made the tables ~25% larger and
    // config 2 ~3% slower).
    reach = rbeam + 2.0 / (double)a.nside + 1e-5;
    // the ring table reserves per-ring slots for footprints up to its reach
    use_tab = reach <= __ldg(&rt[0].ta);
  }
  if (threadIdx.x == 0) {
    w.hdr = make_int4(0, 0, 0, 0);
    w.ir_lo = 0;
  }
  const VecT* svec = nullptr;
  const float* sbv = nullptr;
  const bool staged = a.beam_stage != 0;
  if (staged) {
    const size_t off = spin2_header_bytes(hdr_rings) + (((size_t)a.tab_cap * sizeof(TabT) + 15) & ~size_t(15));
    stage_beam<VecT, NT>(a, smem_raw + off, &s_bar, svec, sbv);
  }
  // one thread derives each sample's rotation and boresight, one sample ahead:
  // the last thread, which has the fewest beam pixels when S is not a multiple
  // of the CTA size
  constexpr int kRotThread = NT - 1;
  constexpr int kRotWarp = NW - 1;
  __shared__ RawFields s_raw;
  if (threadIdx.x == kRotThread && t_begin < t_end)
    write_block<PM>(a, GlobalFields<PM>{a, t_begin * tile}, HAS_QU, s_blk[0]);
  int slot = 0;
  unsigned long long nerr = 0;
  long long prev = -1;
  const int S = (int)a.S;
  for (long long t = t_begin; t < t_end; t += t_step)
  for (long long b = t * tile, b_stop = min(a.B, (t + 1) * tile); b < b_stop; ++b) {
    __syncthreads();  // previous sample is done with the table, its partial sums and its block
    const SampleBlock* sb = &s_blk[slot];
    // the next sample: its pointing fields start on their way to shared memory
    // now, and the last thread turns them into its block after its pixels
    long long bn = b + 1, tn = t;
    if (bn >= b_stop) {
      tn = t + t_step;
      bn = tn * tile;
    }
    const bool has_next = tn < t_end && bn < a.B;
    if (warp == kRotWarp && has_next) prefetch_fields<PM>(a, bn, s_raw, lane);
    if (prev >= 0 && threadIdx.x == 0) flush_sample<kSumLanes / 32>(a, s_red, prev);
    if (use_tab) {
      if (threadIdx.x < kSetupThreads) {
        // footprint window of this sample (same values in every setup thread)
        double ux, uy, uz;
        rotate_block_f64(*sb, cx, cy, cz, ux, uy, uz);
        footprint_window(a, rt, w, ux, uy, uz, reach);
      }
      __syncthreads();
      const int4 hdr = w.hdr;
      const int ntab = hdr.z, nwin = hdr.y;
      const Bore bo{sb->bz, sb->bsth, sb->bphi};
      for (int e = threadIdx.x; e < ntab; e += NT) {
        int lo = 0, hi = nwin - 1;  // last window ring with off <= e
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (w.ring[mid].x <= e)
            lo = mid;
          else
            hi = mid - 1;
        }
        const int4 wr = w.ring[lo];
        const RingRec* r = rt + w.ir_lo + lo;
        const int n = __ldg(&r->n);
        int ip = wr.y + (e - wr.x);
        if (ip >= n) ip -= n;
        const double phin = __ldg(&r->phi0) + (double)ip * __ldg(&r->dphi);
        double c2, s2;
        spin2_c2s2(__ldg(&r->z), __ldg(&r->sth), phin, bo.z, bo.sth, bo.phi, c2, s2);
        tab[e] = make_tab<TabT>(c2, s2);
      }
    }
    __syncthreads();

    // summation lane l (of kSumLanes) takes the beam pixels l, l + kSumLanes,
    // ...; thread t is lane t + i NT in pass i, so the TOD does not depend on
    // the CTA's thread count
#pragma unroll 1
    for (int pass = 0; pass < kSumLanes / NT; ++pass) {
      const int sl = threadIdx.x + pass * NT;
      Acc acc;
      for (int s = sl; s < S; s += kSumLanes) {
        VecT v0, v1, v2;
        float bvf;
        if (staged) {
          v0 = svec[3 * s];
          v1 = svec[3 * s + 1];
          v2 = svec[3 * s + 2];
          bvf = sbv[s];
        } else {
          const VecT* v = static_cast<const VecT*>(a.vec) + 3 * s;
          v0 = __ldg(v);
          v1 = __ldg(v + 1);
          v2 = __ldg(v + 2);
          bvf = __ldg(a.beam + s);
        }
        double vx, vy, vz;
        rotate_block(sb, v0, v1, v2, vx, vy, vz);
        double phi_w = atan2(vy, vx);
        if (phi_w < 0.0) phi_w += kTwoPi;
        if (fast && isfinite(vx) && isfinite(vy) && isfinite(vz)) {
          eval_fast<MODE, HAS_QU, MapT, LAYOUT>(a, sb, rt, w, tab, vx, vy, vz, phi_w, bvf, acc);
        } else if constexpr (MODE == TODGPU_BILINEAR) {
          const Contrib r =
              rt != nullptr
                  ? eval_generic<MODE, HAS_QU, MapT>(a, sb, TableRings{rt}, w, tab, vx, vy, vz, phi_w, bvf)
                  : eval_generic<MODE, HAS_QU, MapT>(a, sb, DirectRings{a.nside, a.npix}, w, tab, vx, vy, vz, phi_w,
                                                     bvf);
          if (r.err) {
            ++nerr;
          } else {
#pragma unroll
            for (int c = 0; c < 4; ++c)
              if (c < a.C) acc.add(c, r.v[c]);
          }
        } else if (rt != nullptr) {
          eval_generic_into<MODE, HAS_QU, MapT>(a, sb, TableRings{rt}, w, tab, vx, vy, vz, phi_w, bvf, acc, nerr);
        } else {
          eval_generic_into<MODE, HAS_QU, MapT>(a, sb, DirectRings{a.nside, a.npix}, w, tab, vx, vy, vz, phi_w, bvf,
                                                acc, nerr);
        }
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= a.C) break;
        const double v = warp_sum(acc.total(c));
        if (lane == 0) s_red[(sl >> 5) * 4 + c] = v;
      }
    }
    // the next sample's rotation into the other block (read after the next barrier)
    if (warp == kRotWarp && has_next) {
      asm volatile("cp.async.wait_all;" ::: "memory");
      __syncwarp();
      if (lane == 31) write_block<PM>(a, SharedFields<PM>{a, s_raw}, HAS_QU, s_blk[slot ^ 1]);
    }
    slot ^= 1;
    prev = b;
  }
  __syncthreads();
  if (prev >= 0 && threadIdx.x == 0) flush_sample<kSumLanes / 32>(a, s_red, prev);
  if (a.err != nullptr) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nerr += __shfl_xor_sync(0xffffffffu, nerr, o);
    if (lane == 0 && nerr) atomicAdd(a.err, nerr);
  }
  __syncthreads();  // the partial sums, tables and blocks may be reused by the next job
}

template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) gather_accum_kernel(const KArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_red[(kSumLanes / 32) * 4];
  run_samples<MODE, HAS_QU, MapT, PM, LAYOUT, NT>(a, blockIdx.x, a.B, gridDim.x, 1, smem_raw, s_red);
}

// Many jobs (detectors: each its own beam, pointing, output and length) in
// one persistent launch.  Job j's samples form tiles of `tile` samples; the
// tiles of all jobs are numbered job by job (tiles_before[j] = tiles of jobs
// 0..j-1) and CTA k takes tiles k, k + G, k + 2G, ... (G = grid size), as one
// launch per job with its samples interleaved over the CTAs would, without a
// launch boundary between jobs.  CTAs running at the same time then work on
// neighbouring samples of one job (the same sky region, shared in L2), and
// every CTA gets an equal share of every job whatever its beam size.  `tile`
// sets how many consecutive samples a CTA takes at a time.  The descriptors
// travel in the kernel parameters; each CTA copies the current job's into
// shared memory, so that the sample loop reads its fields with plain shared
// loads rather than parameter loads at a job index known only at run time
// (5% of the batched launch).
constexpr int kMaxBatchJobs = 96;
struct BatchParams {
  int njobs;
  long long tile;
  long long tiles_before[kMaxBatchJobs + 1];
  KArgs job[kMaxBatchJobs];
};

template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) gather_batched_kernel(const __grid_constant__ BatchParams p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_red[(kSumLanes / 32) * 4];
  __shared__ __align__(16) KArgs s_job;
  const long long G = gridDim.x, k = blockIdx.x;
  for (int j = 0; j < p.njobs; ++j) {
    const long long ntiles = p.tiles_before[j + 1] - p.tiles_before[j];
    // first tile of job j that falls to this CTA: global index = k (mod G)
    const long long t0 = ((k - p.tiles_before[j]) % G + G) % G;
    if (t0 < ntiles) {
      __syncthreads();
      if (threadIdx.x < (int)(sizeof(KArgs) / 8))
        reinterpret_cast<unsigned long long*>(&s_job)[threadIdx.x] =
            reinterpret_cast<const unsigned long long*>(&p.job[j])[threadIdx.x];
      __syncthreads();
      run_samples<MODE, HAS_QU, MapT, PM, LAYOUT, NT>(s_job, t0, ntiles, G, p.tile, smem_raw, s_red);
    }
  }
}

// ---------------------------------------------------------------------------
// Host-side launch templates.
// ---------------------------------------------------------------------------

inline int sm_count() {
  static int count = 0;
  static std::once_flag once;
  std::call_once(once, [] {
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
    if (count <= 0) count = 148;
  });
  return count;
}

struct LaunchInfo {
  int blocks_per_sm = 0;
  size_t smem = 0;  // dynamic shared memory blocks_per_sm was computed for
  bool configured = false;
};

// Shared memory per SM on B200 and what the driver keeps per CTA; the
// kernels' static shared memory (partial sums, rotation slots) stays well
// under the 2 KiB margin below.
constexpr size_t kSmemPerSM = 228 * 1024;
constexpr size_t kSmemPerCTAReserved = 1024;
constexpr size_t kStaticSmemMargin = 2048;

#ifndef TODGPU_CTA_THREADS
#define TODGPU_CTA_THREADS 256
#endif
constexpr int kNT = TODGPU_CTA_THREADS;  // threads per CTA

// CTAs per SM the register budget is sized for: 4 (64 registers) for the
// nearest mode and packed maps, where the fourth CTA measured 3-5% faster; 3
// (80 registers) for bilinear on planar maps, where it gained nothing and the
// extra spilling doubled the local-memory write-back to DRAM.
template <int MODE, typename MapT>
constexpr int min_blocks() {
#ifdef TODGPU_CTA_MINB
  return TODGPU_CTA_MINB;
#else
  return (MODE == TODGPU_NEAREST || MapTraits<MapT>::packed) ? 4 : 3;
#endif
}

// Dynamic shared memory a CTA may take while MINB CTAs still fit on an SM.
template <int MINB>
constexpr size_t cta_smem_budget() {
  return kSmemPerSM / MINB - kSmemPerCTAReserved - kStaticSmemMargin;
}

// Window rings a launch's table header reserves.  A request of N slots is a
// footprint disc of at most N / 3.2 pixels (the request of kernels.table_slots
// is 1.05 x (1.02 x 3 (r nside)^2 + 3 per ring) + 32 for a disc of radius r),
// so r nside <= sqrt(N / 3.2), and such a disc crosses at most 3 r nside + 4
// rings of the RING scheme (ring spacing at least 2 / (3 nside) in colatitude,
// plus the rings either side); the default table reserves kRingCap.  The
// header then takes 32 + 16 x rings bytes instead of 3 KiB, and the shared
// memory left goes to L1.
inline int ring_cap_for(int requested) {
  if (requested <= 0) return kRingCap;
  return std::min(kRingCap, (int)std::ceil(3.0 * std::sqrt(requested / 3.2)) + 6);
}

// Spin-2 table slots of a launch: the caller's request, else 32 KiB (2048
// float64 or 4096 float32 pairs); never more than each of MINB CTAs can hold
// in an SM's shared memory beside the table header.
template <typename TabT, int MINB>
int max_table_slots(int ring_cap) {
  return (int)((cta_smem_budget<MINB>() - spin2_header_bytes(ring_cap)) / sizeof(TabT));
}
constexpr size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

// Modes whose launches stage the beam in shared memory when it fits: bilinear
// (config 2 in 256-thread CTAs: +5%; its 128-thread CTAs have no room for
// the beam beside the table); nearest reads one stencil pixel per beam pixel
// and gains more from the shared memory left to L1 (1% faster without).
template <int MODE>
constexpr bool stage_beam_mode() {
  return MODE == TODGPU_BILINEAR;
}

template <typename TabT, int MINB>
int table_slots(int requested, int ring_cap) {
  constexpr int kCap = (int)(kTabCapDefault * sizeof(double2) / sizeof(TabT));
  return requested > 0 ? std::min(requested, max_table_slots<TabT, MINB>(ring_cap)) : kCap;
}

// Window rings of a launch's table header: fixed in the narrow shape.
template <int NT>
int header_rings(bool table, int requested) {
  if (NT == kNTNarrow) return kRingCapNarrow;
  return table ? ring_cap_for(requested) : 1;  // ring[0] is read (not used) without a window
}

// Once per kernel: allow the largest table; per launch: CTAs per SM for the
// launch's shared memory (recomputed when it changes).
template <int NT, typename Kern>
int configure_launch(Kern kern, LaunchInfo& info, std::mutex& mu, size_t smem, int& blocks_per_sm) {
  std::lock_guard<std::mutex> lock(mu);
  if (!info.configured) {
    // the largest dynamic shared memory a CTA of this kernel can have
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
    if (e != cudaSuccess) return cuda_fail(e, "kernel shared-memory attributes");
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
    info.configured = true;
    info.blocks_per_sm = 0;
  }
  if (info.blocks_per_sm == 0 || info.smem != smem) {
    int nb = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, NT, smem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    info.blocks_per_sm = std::max(nb, 1);
    info.smem = smem;
  }
  blocks_per_sm = info.blocks_per_sm;
  return TODGPU_OK;
}

// Two CTA shapes.  Wide: kNT (256) threads, min_blocks() CTAs per SM, room
// for the default 32 KiB spin-2 table and the staged beam.  Narrow: 128
// threads, 8 CTAs per SM at 64 registers, for launches whose requested table
// fits an eighth of an SM's shared memory beside the shape's 80-ring header
// (config 2: 820 slots of 16 B): with more CTAs per SM, the per-sample setup
// and barriers of one CTA overlap the pixel loops of more others (config 2
// bilinear +12%, nearest +7%, although the beam no longer fits beside the
// table).  Larger footprints (config 3: 3.2k slots) keep the wide shape: in
// the narrow one their tables would not fit and their samples would fall back
// to direct spin-2 evaluation.  The TOD is the same bit for bit in either
// shape (kSumLanes).
template <typename TabT>
bool narrow_fits(int requested) {
  return requested > 0 && ring_cap_for(requested) <= kRingCapNarrow &&
         requested <= max_table_slots<TabT, kMinbNarrow>(kRingCapNarrow);
}

template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT, int NT, int MINB>
int launch_gather_shape(KArgs k, cudaStream_t stream) {
  auto kern = gather_accum_kernel<MODE, HAS_QU, MapT, PM, LAYOUT, NT, MINB>;
  static LaunchInfo info;
  static std::mutex mu;
  using TabT = typename MapTraits<MapT>::Tab;
  const bool tab = HAS_QU && k.ring_table != nullptr;
  k.ring_cap = header_rings<NT>(tab, k.tab_req);
  const int tab_cap = tab ? table_slots<TabT, MINB>(k.tab_req, k.ring_cap) : 0;
  const size_t tab_end = spin2_header_bytes(k.ring_cap) + align16(sizeof(TabT) * (size_t)tab_cap);
  const size_t stage = beam_stage_bytes(k.S, PM == kParamsRef32 ? sizeof(float) : sizeof(double));
  k.beam_stage = (stage_beam_mode<MODE>() && k.flags_stage && tab_end + stage <= cta_smem_budget<MINB>()) ? 1 : 0;
  const size_t smem = tab_end + (k.beam_stage ? stage : 0);
  int blocks_per_sm = 0;
  const int rc = configure_launch<NT>(kern, info, mu, smem, blocks_per_sm);
  if (rc != TODGPU_OK) return rc;
  k.tab_cap = tab_cap;
  const long long max_blocks = (long long)sm_count() * blocks_per_sm;
  const int grid = (int)std::max(1LL, std::min(k.B, max_blocks));
  kern<<<grid, NT, smem, stream>>>(k);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "gather_accum_kernel launch");
  return TODGPU_OK;
}

template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT>
int launch_gather(KArgs k, cudaStream_t stream) {
  using TabT = typename MapTraits<MapT>::Tab;
  if (!k.flags_wide && narrow_fits<TabT>(k.tab_req))
    return launch_gather_shape<MODE, HAS_QU, MapT, PM, LAYOUT, kNTNarrow, kMinbNarrow>(k, stream);
  return launch_gather_shape<MODE, HAS_QU, MapT, PM, LAYOUT, kNT, min_blocks<MODE, MapT>()>(k, stream);
}

static_assert(sizeof(BatchParams) <= 32000, "batched descriptors must fit the kernel parameter space");
static_assert(sizeof(KArgs) % 8 == 0 && sizeof(KArgs) / 8 <= kNTNarrow, "KArgs copied as 8-byte words, one per thread");

// Batched launch: descriptors of up to kMaxBatchJobs jobs per launch, in one
// CTA shape: narrow when every job allows it and the table size the launch
// takes (the largest any job asks for; a job asking for the default makes it
// the default) fits it.
template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT, int NT, int MINB>
int launch_batched_shape(BatchParams& bp, bool any_table, int req, bool any_default, cudaStream_t stream) {
  auto kern = gather_batched_kernel<MODE, HAS_QU, MapT, PM, LAYOUT, NT, MINB>;
  static LaunchInfo info;
  static std::mutex mu;
  using TabT = typename MapTraits<MapT>::Tab;
  const int ring_cap = header_rings<NT>(HAS_QU && any_table, any_default ? 0 : req);
  const int tab_cap = (HAS_QU && any_table) ? table_slots<TabT, MINB>(any_default ? 0 : req, ring_cap) : 0;
  const size_t tab_end = spin2_header_bytes(ring_cap) + align16(sizeof(TabT) * (size_t)tab_cap);
  // one shared region for every job's beam: sized for the largest
  size_t stage = 0;
  bool want_stage = true;
  for (int j = 0; j < bp.njobs; ++j) {
    stage = std::max(stage, beam_stage_bytes(bp.job[j].S, PM == kParamsRef32 ? sizeof(float) : sizeof(double)));
    want_stage = want_stage && bp.job[j].flags_stage;
  }
  const int staged = (stage_beam_mode<MODE>() && want_stage && tab_end + stage <= cta_smem_budget<MINB>()) ? 1 : 0;
  const size_t smem = tab_end + (staged ? stage : 0);
  int blocks_per_sm = 0;
  const int rc = configure_launch<NT>(kern, info, mu, smem, blocks_per_sm);
  if (rc != TODGPU_OK) return rc;
  for (int j = 0; j < bp.njobs; ++j) {
    bp.job[j].tab_cap = tab_cap;
    bp.job[j].ring_cap = ring_cap;
    bp.job[j].beam_stage = staged;
  }
  const long long T = bp.tiles_before[bp.njobs];
  if (T == 0) return TODGPU_OK;
  const long long max_blocks = (long long)sm_count() * blocks_per_sm;
  const int grid = (int)std::max(1LL, std::min(T, max_blocks));
  kern<<<grid, NT, smem, stream>>>(bp);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "gather_batched_kernel launch");
  return TODGPU_OK;
}

template <int MODE, bool HAS_QU, typename MapT, int PM, int LAYOUT>
int launch_batched(BatchParams& bp, bool any_table, cudaStream_t stream) {
  using TabT = typename MapTraits<MapT>::Tab;
  int req = 0;
  bool any_default = false, any_wide = false;
  for (int j = 0; j < bp.njobs; ++j) {
    req = std::max(req, bp.job[j].tab_req);
    any_default = any_default || bp.job[j].tab_req == 0;
    any_wide = any_wide || bp.job[j].flags_wide;
  }
  if (!any_wide && !any_default && narrow_fits<TabT>(req))
    return launch_batched_shape<MODE, HAS_QU, MapT, PM, LAYOUT, kNTNarrow, kMinbNarrow>(bp, any_table, req, false,
                                                                                        stream);
  return launch_batched_shape<MODE, HAS_QU, MapT, PM, LAYOUT, kNT, min_blocks<MODE, MapT>()>(bp, any_table, req,
                                                                                           any_default, stream);
}

template <int MODE, typename MapT, int PM>
int dispatch_batched_qu(BatchParams& bp, bool has_qu, bool iqu, bool any_table, cudaStream_t s) {
  if (has_qu && iqu) return launch_batched<MODE, true, MapT, PM, kLayoutIQU>(bp, any_table, s);
  return has_qu ? launch_batched<MODE, true, MapT, PM, kLayoutGeneric>(bp, any_table, s)
                : launch_batched<MODE, false, MapT, PM, kLayoutGeneric>(bp, any_table, s);
}

template <int MODE, typename MapT, int PM>
int dispatch_qu(const KArgs& k, bool has_qu, cudaStream_t s) {
  if (has_qu && k.C == 3 && k.c_q == 1 && k.c_u == 2) return launch_gather<MODE, true, MapT, PM, kLayoutIQU>(k, s);
  return has_qu ? launch_gather<MODE, true, MapT, PM, kLayoutGeneric>(k, s)
                : launch_gather<MODE, false, MapT, PM, kLayoutGeneric>(k, s);
}


// Pointing-mode switch of one map element type (instantiated by gather_map_*.cu).
template <int MODE, typename MapT>
int dispatch_single_pm(const KArgs& k, bool has_qu, int params_dtype, cudaStream_t s) {
  if (params_dtype == TODGPU_F32) return dispatch_qu<MODE, MapT, kParamsRef32>(k, has_qu, s);
  if (params_dtype == TODGPU_F64) return dispatch_qu<MODE, MapT, kParamsF64>(k, has_qu, s);
  return dispatch_qu<MODE, MapT, kAngles>(k, has_qu, s);
}

template <int MODE, typename MapT>
int dispatch_batched_pm(BatchParams& bp, bool has_qu, bool iqu, bool any_table, int params_dtype, cudaStream_t s) {
  if (params_dtype == TODGPU_F32) return dispatch_batched_qu<MODE, MapT, kParamsRef32>(bp, has_qu, iqu, any_table, s);
  if (params_dtype == TODGPU_F64) return dispatch_batched_qu<MODE, MapT, kParamsF64>(bp, has_qu, iqu, any_table, s);
  return dispatch_batched_qu<MODE, MapT, kAngles>(bp, has_qu, iqu, any_table, s);
}

// Entry points of the per-map-type translation units.
#define TODGPU_DECLARE_MAP_DISPATCH(NAME)                                                                   \
  int dispatch_single_##NAME(const KArgs& k, int interp, bool has_qu, int params_dtype, cudaStream_t s);   \
  int dispatch_batched_##NAME(BatchParams& bp, int interp, bool has_qu, bool iqu, bool any_table,          \
                              int params_dtype, cudaStream_t s);
TODGPU_DECLARE_MAP_DISPATCH(f64)
TODGPU_DECLARE_MAP_DISPATCH(f32)
TODGPU_DECLARE_MAP_DISPATCH(pf32)
TODGPU_DECLARE_MAP_DISPATCH(pbf16)
TODGPU_DECLARE_MAP_DISPATCH(pf64)
#undef TODGPU_DECLARE_MAP_DISPATCH

#define TODGPU_DEFINE_MAP_DISPATCH(NAME, MAPT)                                                             \
  int dispatch_single_##NAME(const KArgs& k, int interp, bool has_qu, int params_dtype, cudaStream_t s) {  \
    return interp == TODGPU_BILINEAR ? dispatch_single_pm<TODGPU_BILINEAR, MAPT>(k, has_qu, params_dtype, s) \
                                     : dispatch_single_pm<TODGPU_NEAREST, MAPT>(k, has_qu, params_dtype, s);  \
  }                                                                                                        \
  int dispatch_batched_##NAME(BatchParams& bp, int interp, bool has_qu, bool iqu, bool any_table,          \
                              int params_dtype, cudaStream_t s) {                                          \
    return interp == TODGPU_BILINEAR                                                                       \
               ? dispatch_batched_pm<TODGPU_BILINEAR, MAPT>(bp, has_qu, iqu, any_table, params_dtype, s)   \
               : dispatch_batched_pm<TODGPU_NEAREST, MAPT>(bp, has_qu, iqu, any_table, params_dtype, s);   \
  }

}  // namespace todgpu
