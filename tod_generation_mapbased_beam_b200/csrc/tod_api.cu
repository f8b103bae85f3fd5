// tod_api.cu -- the C ABI of include/todgpu.h: argument checks, the ring
// table, the built-in table of the allocation-free entry point, the small
// parity kernels and the map packer.  The gather kernels themselves are
// instantiated in gather_map_*.cu.
#include "gather_impl.cuh"

namespace todgpu {

thread_local std::string g_last_error;

// Ring table: record ir (1 .. 4 nside - 1) of every ring; record 0 holds
// nside and the reach.  cap_r bounds the pixels of ring r inside any disc of
// radius `reach`: a disc meets the latitude of the ring in a longitude
// interval of half-width at most asin(sin(reach) / sin(theta_r)), or the
// whole ring when the disc can contain the pole.
__global__ void ring_table_kernel(long long nside, double reach, RingRec* t, bool reach_from_header) {
  const long long nrings = 4 * nside - 1;
  const long long npix = 12 * nside * nside;
  if (reach_from_header) reach = t[0].ta;
  for (long long ir = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; ir <= nrings;
       ir += (long long)gridDim.x * blockDim.x) {
    const RingInfo ri = hp_ring_info(nside, ir, npix);
    RingRec r;
    r.z = hp_ring_z(nside, ir);
    r.ta = acos(r.z);
    r.sth = sqrt(max0(1.0 - r.z * r.z));
    r.phi0 = ri.phi0;
    r.dphi = ri.dphi;
    r.first = ri.first;
    r.n = (int)ri.n;
    int cap = (int)ri.n;
    if (reach < r.ta && reach < kPi - r.ta) {
      const double x = sin(reach) / r.sth;
      if (x < 1.0) {
        const double half = asin(x);
        const long long c = 2 * (long long)ceil(half / ri.dphi) + 5;
        cap = (int)min(c, ri.n);
      }
    }
    r.cap = cap;
    r.unused = 0;
    r.first32 = (int)ri.first;
    r.inv_dphi = 1.0 / ri.dphi;
    r.inv_dta = ir < nrings ? 1.0 / (acos(hp_ring_z(nside, ir + 1)) - r.ta) : 0.0;
    t[ir] = r;
  }
  if (!reach_from_header && blockIdx.x == 0 && threadIdx.x == 0) {
    RingRec h;
    h.z = (double)nside;
    h.ta = reach;
    h.sth = 0.0;
    h.phi0 = 0.0;
    h.dphi = 0.0;
    h.first = 0;
    h.n = 0;
    h.cap = 0;
    h.first32 = 0;
    h.unused = 0;
    h.inv_dphi = 0.0;
    h.inv_dta = 0.0;
    t[0] = h;
  }
}

// ---------------------------------------------------------------------------
// Small parity kernels (one thread per element).
// ---------------------------------------------------------------------------

template <int PM>
__global__ void stencil_kernel(const KArgs a, long long* pix, double* wgt) {
  const long long BS = a.B * a.S;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < BS;
       n += (long long)gridDim.x * blockDim.x) {
    const long long b = n / a.S, s = n - b * a.S;
    const SampleRot rot = load_rot<PM>(a, b);
    double vx, vy, vz;
    if constexpr (PM != kParamsRef32) {
      const double* v = static_cast<const double*>(a.vec) + 3 * s;
      rot_f64(rot, v[0], v[1], v[2], vx, vy, vz);
    } else {
      const float* v = static_cast<const float*>(a.vec) + 3 * s;
      rot_ref32(rot, v[0], v[1], v[2], vx, vy, vz);
    }
    const double z = clamp1(vz);
    double phi_w = atan2(vy, vx);
    if (phi_w < 0.0) phi_w += kTwoPi;
    hp_stencil(a.nside, z, phi_w, DirectRings{a.nside, a.npix},
               [&](int k, long long p, double wk, long long, long long, long long, double, double) {
                 pix[k * BS + n] = p;
                 wgt[k * BS + n] = wk;
               });
  }
}

// hp.get_interp_weights on (theta, phi): theta-based weights
// (numba_healpy.py:120-236).
__global__ void interp_weights_kernel(long long nside, const double* theta, const double* phi, long long N,
                                      long long* pix, double* wgt) {
  const long long npix = 12 * nside * nside;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double th = theta[i], ph = phi[i];
    const double z = cos(th);
    const long long ir_above = hp_ring_above(nside, z);
    const long long ir_below = wrap_add(ir_above, 1);
    long long p[4];
    double w[4];
    if (ir_above == 0) {
      RingInfo ra = hp_ring_info(nside, 1, npix);
      double tw = py_fmod_pos((ph - ra.phi0) / ra.dphi, (double)ra.n);
      long long ip = py_int(tw);
      double frac = tw - (double)ip;
      long long ip2 = py_imod(wrap_add(ip, 1), ra.n);
      p[2] = wrap_add(ra.first, ip);
      p[3] = ra.first + ip2;
      p[0] = py_imod(wrap_add(ip, 2), ra.n);
      p[1] = py_imod(ip2 + 2, ra.n);
      double ta = acos(hp_ring_z(nside, 1));
      double wt = th / ta;
      double nf = (1.0 - wt) * 0.25;
      w[0] = nf;
      w[1] = nf;
      w[2] = (1.0 - frac) * wt + nf;
      w[3] = frac * wt + nf;
    } else if (ir_below == 4 * nside) {
      const long long ir_last = 4 * nside - 1;
      RingInfo ra = hp_ring_info(nside, ir_last, npix);
      double tw = py_fmod_pos((ph - ra.phi0) / ra.dphi, (double)ra.n);
      long long ip = py_int(tw);
      double frac = tw - (double)ip;
      long long ip2 = py_imod(wrap_add(ip, 1), ra.n);
      p[0] = wrap_add(ra.first, ip);
      p[1] = ra.first + ip2;
      p[2] = py_imod(wrap_add(ip, 2), ra.n) + ra.first;
      p[3] = py_imod(ip2 + 2, ra.n) + ra.first;
      double ta = acos(hp_ring_z(nside, ir_last));
      double ws = (th - ta) / (kPi - ta);
      double sf = ws * 0.25;
      w[0] = (1.0 - frac) * (1.0 - ws) + sf;
      w[1] = frac * (1.0 - ws) + sf;
      w[2] = sf;
      w[3] = sf;
    } else {
      double ta = acos(hp_ring_z(nside, ir_above));
      double tb = acos(hp_ring_z(nside, ir_below));
      double wb = (th - ta) / (tb - ta);
      double wa = 1.0 - wb;
      RingInfo ra = hp_ring_info(nside, ir_above, npix);
      double tw = py_fmod_pos((ph - ra.phi0) / ra.dphi, (double)ra.n);
      long long ia = py_int(tw);
      double fa = tw - (double)ia;
      p[0] = wrap_add(ra.first, ia);
      p[1] = ra.first + py_imod(wrap_add(ia, 1), ra.n);
      w[0] = wa * (1.0 - fa);
      w[1] = wa * fa;
      RingInfo rb = hp_ring_info(nside, ir_below, npix);
      tw = py_fmod_pos((ph - rb.phi0) / rb.dphi, (double)rb.n);
      long long ib = py_int(tw);
      double fb = tw - (double)ib;
      p[2] = wrap_add(rb.first, ib);
      p[3] = rb.first + py_imod(wrap_add(ib, 1), rb.n);
      w[2] = wb * (1.0 - fb);
      w[3] = wb * fb;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      pix[k * N + i] = p[k];
      wgt[k * N + i] = w[k];
    }
  }
}

__global__ void ang2pix_kernel(long long nside, const double* theta, const double* phi, long long N, long long* out) {
  const long long npix = 12 * nside * nside;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double z = cos(theta[i]);
    double phi_w = fmod(phi[i], kTwoPi);
    if (phi_w != 0.0) {
      if (phi_w < 0.0) phi_w += kTwoPi;
    } else {
      phi_w = 0.0;
    }
    out[i] = hp_nearest(nside, z, sin(theta[i]), phi_w, DirectRingsNoAcos{nside, npix}).pix;
  }
}

__global__ void pix2ang_kernel(long long nside, const long long* pixs, long long N, double* theta, double* phi) {
  const long long npix = 12 * nside * nside;
  const long long ncap = 2 * nside * (nside - 1);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const long long pix = pixs[i];
    long long iring, ip_in;
    if (pix < ncap) {
      iring = py_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)pix)));
      ip_in = pix - 2 * iring * (iring - 1);
    } else if (pix < npix - ncap) {
      const long long ip = pix - ncap;
      iring = ip / (4 * nside) + nside;
      ip_in = ip % (4 * nside);
    } else {
      const long long ips = npix - pix - 1;
      const long long irs = py_int(0.5 * (1.0 + sqrt(1.0 + 2.0 * (double)ips)));
      iring = 4 * nside - irs;
      ip_in = pix - (npix - 2 * irs * (irs + 1));
    }
    const RingInfo r = hp_ring_info(nside, iring, npix);
    phi[i] = r.phi0 + (double)ip_in * r.dphi;
    theta[i] = acos(hp_ring_z(nside, iring));
  }
}

__global__ void spin2_kernel(const double* zp, const double* sp, const double* pp, const double* zq, const double* sq,
                             const double* pq, long long N, double* c2d, double* s2d) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    double c, s;
    spin2_c2s2(zp[i], sp[i], pp[i], zq[i], sq[i], pq[i], c, s);
    c2d[i] = c;
    s2d[i] = s;
  }
}

// ---------------------------------------------------------------------------
// Built-in ring table for callers that cannot allocate device memory.
// ---------------------------------------------------------------------------

// Largest nside the built-in table holds: 4 * 4096 records of 80 bytes = 1.25 MiB,
// resident on every GPU that loads the library until the process exits.
constexpr long long kStaticMaxNside = 4096;
static __device__ __align__(256) RingRec g_static_ring_table[4 * kStaticMaxNside];

// Header of a table built from the beam on the device: the footprint reach the
// gather kernel derives from the same beam (same code, plus a hair of margin).
template <int PM>
__global__ void __launch_bounds__(kNTStatic) static_reach_kernel(const KArgs a, RingRec* t) {
  __shared__ double s_red[(kNTStatic / 32) * 4];
  double cx, cy, cz, rbeam;
  beam_extent<PM, kNTStatic>(a, s_red, cx, cy, cz, rbeam);
  if (threadIdx.x == 0) {
    RingRec h;
    h.z = (double)a.nside;
    h.ta = rbeam + 3.0 / (double)a.nside + 1e-5 + 1e-9;
    h.sth = 0.0;
    h.phi0 = 0.0;
    h.dphi = 0.0;
    h.first = 0;
    h.n = 0;
    h.cap = 0;
    h.first32 = 0;
    h.unused = 0;
    h.inv_dphi = 0.0;
    h.inv_dta = 0.0;
    t[0] = h;
  }
}

// Planar (C, N) float/double map -> one float64 record of 4 components per
// pixel (missing components are 0), as two 16-byte stores.
template <typename SrcT>
__global__ void pack_map_f64_kernel(const SrcT* src, int C, long long N, long long stride, void* out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = 0; c < C; ++c) v[c] = (double)src[(long long)c * stride + p];
    double2* o = static_cast<double2*>(out) + 2 * p;
    o[0] = make_double2(v[0], v[1]);
    o[1] = make_double2(v[2], v[3]);
  }
}

// Planar (C, N) float/double map -> one record per pixel of 4 components
// (float32 or bfloat16, round to nearest even; missing components are 0).
template <typename SrcT, bool BF16>
__global__ void pack_map_kernel(const SrcT* src, int C, long long N, long long stride, void* out) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
    float v[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < C; ++c) v[c] = (float)src[(long long)c * stride + p];
    if constexpr (BF16) {
      __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]);
      __nv_bfloat162 hi = __floats2bfloat162_rn(v[2], v[3]);
      uint2 r;
      r.x = *reinterpret_cast<unsigned*>(&lo);
      r.y = *reinterpret_cast<unsigned*>(&hi);
      static_cast<uint2*>(out)[p] = r;
    } else {
      static_cast<float4*>(out)[p] = make_float4(v[0], v[1], v[2], v[3]);
    }
  }
}

// FP64 pipe throughput probe: 8 independent FMA chains per thread, so the
// pipe, not latency, bounds it.  flops = 2 * 8 * iters per thread.
__global__ void fp64_probe_kernel(int iters, double seed, double* out) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
         a7 = a0 + 7;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, m, c);
    a1 = fma(a1, m, c);
    a2 = fma(a2, m, c);
    a3 = fma(a3, m, c);
    a4 = fma(a4, m, c);
    a5 = fma(a5, m, c);
    a6 = fma(a6, m, c);
    a7 = fma(a7, m, c);
  }
  const double v = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (v == 12345.678) out[blockIdx.x] = v;  // keeps the chains alive; never true in practice
}


// Map element type switch of the single and batched launches.
static int dispatch_types(const KArgs& k, int interp, bool has_qu, int map_dtype, int params_dtype, cudaStream_t s) {
  switch (map_dtype) {
    case TODGPU_PACKED_F32: return dispatch_single_pf32(k, interp, has_qu, params_dtype, s);
    case TODGPU_PACKED_BF16: return dispatch_single_pbf16(k, interp, has_qu, params_dtype, s);
    case TODGPU_PACKED_F64: return dispatch_single_pf64(k, interp, has_qu, params_dtype, s);
    case TODGPU_F32: return dispatch_single_f32(k, interp, has_qu, params_dtype, s);
    default: return dispatch_single_f64(k, interp, has_qu, params_dtype, s);
  }
}

static int dispatch_batched(BatchParams& bp, int interp, bool has_qu, bool iqu, bool any_table, int map_dtype,
                            int params_dtype, cudaStream_t s) {
  switch (map_dtype) {
    case TODGPU_PACKED_F32: return dispatch_batched_pf32(bp, interp, has_qu, iqu, any_table, params_dtype, s);
    case TODGPU_PACKED_BF16: return dispatch_batched_pbf16(bp, interp, has_qu, iqu, any_table, params_dtype, s);
    case TODGPU_PACKED_F64: return dispatch_batched_pf64(bp, interp, has_qu, iqu, any_table, params_dtype, s);
    case TODGPU_F32: return dispatch_batched_f32(bp, interp, has_qu, iqu, any_table, params_dtype, s);
    default: return dispatch_batched_f64(bp, interp, has_qu, iqu, any_table, params_dtype, s);
  }
}

static int check_common(const todgpu_gather_args* a, bool need_map) {
  if (a == nullptr) return fail(TODGPU_EINVAL, "args is NULL");
  if (a->abi_version != TODGPU_ABI_VERSION)
    return fail(TODGPU_EABI, "abi_version " + std::to_string(a->abi_version) + " != " +
                                 std::to_string(TODGPU_ABI_VERSION));
  if (a->nside < 1 || a->nside > kMaxNside)
    return fail(TODGPU_ENSIDE, "nside " + std::to_string(a->nside) + " outside [1, 16384]");
  if (a->B < 0 || a->S < 0) return fail(TODGPU_ESHAPE, "negative B or S");
  if (a->S > (1LL << 29)) return fail(TODGPU_ESHAPE, "S above 2^29 beam pixels");
  if (a->tab_slots < 0) return fail(TODGPU_EINVAL, "tab_slots must be >= 0");
  if (a->params_dtype != TODGPU_F32 && a->params_dtype != TODGPU_F64 && a->params_dtype != TODGPU_ANGLES)
    return fail(TODGPU_EDTYPE, "params_dtype must be TODGPU_F32, TODGPU_F64 or TODGPU_ANGLES");
  if (a->B > 0 && a->S > 0) {
    const uintptr_t vec_align = a->params_dtype == TODGPU_F32 ? 3 : 7;
    if (((uintptr_t)a->vec_orig & vec_align) != 0 || ((uintptr_t)a->beam_vals & 3) != 0)
      return fail(TODGPU_EINVAL, "vec_orig and beam_vals must be aligned to their element size");
    if (a->params_dtype == TODGPU_ANGLES) {
      if (!a->vec_orig || !a->theta || !a->phi || !a->psi) return fail(TODGPU_EINVAL, "NULL pointing array");
      if (a->angles_dtype != TODGPU_F32 && a->angles_dtype != TODGPU_F64)
        return fail(TODGPU_EDTYPE, "angles_dtype must be TODGPU_F32 or TODGPU_F64");
    } else if (!a->vec_orig || !a->axes || !a->cos_a || !a->sin_a || !a->ax_pts || !a->cos_p || !a->sin_p) {
      return fail(TODGPU_EINVAL, "NULL parameter array");
    }
  }
  if (need_map) {
    if (a->interp != TODGPU_BILINEAR && a->interp != TODGPU_NEAREST)
      return fail(TODGPU_EINVAL, "interp must be TODGPU_BILINEAR or TODGPU_NEAREST");
    if (a->C < 1 || a->C > 4) return fail(TODGPU_ESHAPE, "C must be in [1, 4]");
    if (a->c_q < -1 || a->c_q >= a->C || a->c_u < -1 || a->c_u >= a->C)
      return fail(TODGPU_ESHAPE, "c_q/c_u must be -1 or a component index");
    if (a->c_q >= 0 && a->c_q == a->c_u) return fail(TODGPU_ESHAPE, "c_q == c_u");
    const bool packed = a->map_dtype == TODGPU_PACKED_F32 || a->map_dtype == TODGPU_PACKED_BF16 ||
                        a->map_dtype == TODGPU_PACKED_F64;
    if (a->map_dtype != TODGPU_F32 && a->map_dtype != TODGPU_F64 && !packed)
      return fail(TODGPU_EDTYPE, "map_dtype must be TODGPU_F32, TODGPU_F64 or a TODGPU_PACKED_* type");
    const long long npix = 12 * a->nside * a->nside;
    if (!packed && a->map_stride < npix) return fail(TODGPU_ESHAPE, "map_stride < 12*nside^2");
    if (packed && ((uintptr_t)a->map & (a->map_dtype == TODGPU_PACKED_BF16 ? 7 : 15)) != 0)
      return fail(TODGPU_EINVAL, "packed map must be aligned to 16 bytes (8 for bfloat16 records)");
    if (a->tod_stride < a->B) return fail(TODGPU_ESHAPE, "tod_stride < B");
    if (a->B > 0 && a->S > 0 && (!a->map || !a->tod || !a->beam_vals))
      return fail(TODGPU_EINVAL, "NULL map, tod or beam_vals");
  }
  return TODGPU_OK;
}

static KArgs make_kargs(const todgpu_gather_args* a) {
  KArgs k;
  k.nside = a->nside;
  k.npix = 12 * a->nside * a->nside;
  k.B = a->B;
  k.S = a->S;
  k.C = (int)a->C;
  k.c_q = a->c_q;
  k.c_u = a->c_u;
  k.vec = a->vec_orig;
  k.axes = a->axes;
  k.cos_a = a->cos_a;
  k.sin_a = a->sin_a;
  k.pts = a->ax_pts;
  k.cos_p = a->cos_p;
  k.sin_p = a->sin_p;
  k.bore_phi = a->bore_phi;
  k.theta = a->theta;
  k.phi = a->phi;
  k.psi = a->psi;
  k.angles_f32 = a->angles_dtype == TODGPU_F32 ? 1 : 0;
  {
    // beam centre and its north from (center_phi, center_theta)
    const double st = std::sin(a->center_theta), ct = std::cos(a->center_theta);
    const double sp = std::sin(a->center_phi), cp = std::cos(a->center_phi);
    k.cvx = st * cp;
    k.cvy = st * sp;
    k.cvz = ct;
    k.cnx = cp * ct;
    k.cny = sp * ct;
    k.cnz = -st;
  }
  k.beam = a->beam_vals;
  k.map = a->map;
  k.map_stride = a->map_stride;
  k.tod = a->tod;
  k.tod_stride = a->tod_stride;
  k.err = a->err_count;
  k.ring_table = (a->flags & TODGPU_FLAG_NO_TABLES) ? nullptr : a->ring_table;
  if (k.ring_table != nullptr && (((uintptr_t)k.ring_table & 15) != 0)) k.ring_table = nullptr;
  k.tab_cap = 0;
  k.tab_req = a->tab_slots;
  k.flags_stage = (a->flags & TODGPU_FLAG_NO_BEAM_STAGE) ? 0 : 1;
  k.beam_stage = 0;
  k.flags_wide = (a->flags & TODGPU_FLAG_WIDE_CTAS) ? 1 : 0;
  k.ring_cap = 0;
  return k;
}

static int grid_for(long long n, int threads) {
  long long blocks = (n + threads - 1) / threads;
  return (int)std::max(1LL, std::min(blocks, (long long)sm_count() * 16));
}

}  // namespace todgpu

using namespace todgpu;

extern "C" int todgpu_gather_accum(const todgpu_gather_args* a, void* stream) {
  int rc = check_common(a, true);
  if (rc != TODGPU_OK) return rc;
  if (a->B == 0 || a->S == 0) return TODGPU_OK;
  const KArgs k = make_kargs(a);
  const bool has_qu = (a->c_q >= 0 && a->c_u >= 0);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return dispatch_types(k, a->interp, has_qu, a->map_dtype, a->params_dtype, s);
}

// Device address of the built-in ring table on the current device, looked up
// once per device (cudaGetSymbolAddress with that device current).
static int static_table_ptr(RingRec** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  static std::mutex mu;
  static std::vector<RingRec*> ptrs;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)ptrs.size() <= dev) ptrs.resize(dev + 1, nullptr);
  if (ptrs[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_ring_table);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_ring_table)");
    ptrs[dev] = static_cast<RingRec*>(p);
  }
  *out = ptrs[dev];
  return TODGPU_OK;
}

extern "C" int todgpu_gather_accum_static(const todgpu_gather_args* a, void* stream) {
  int rc = check_common(a, true);
  if (rc != TODGPU_OK) return rc;
  if (a->nside > kStaticMaxNside)
    return fail(TODGPU_ENSIDE, "nside " + std::to_string(a->nside) +
                                   " exceeds 4096, the largest nside of the built-in ring table; use "
                                   "todgpu_gather_accum with a caller-allocated table");
  if (a->B == 0 || a->S == 0) return TODGPU_OK;
  RingRec* t = nullptr;
  rc = static_table_ptr(&t);
  if (rc != TODGPU_OK) return rc;
  KArgs k = make_kargs(a);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool has_qu = (a->c_q >= 0 && a->c_u >= 0);
  if (!(a->flags & TODGPU_FLAG_NO_TABLES)) {
    // every call rebuilds the whole table (header and records) for its own
    // nside and beam, so nothing depends on earlier contents.  Without Q and U
    // the gather reads only the ring records (no spin-2 tables): the header
    // then carries a zero reach.
    if (has_qu) {
      if (a->params_dtype == TODGPU_F32)
        static_reach_kernel<kParamsRef32><<<1, kNTStatic, 0, s>>>(k, t);
      else
        static_reach_kernel<kParamsF64><<<1, kNTStatic, 0, s>>>(k, t);
      ring_table_kernel<<<grid_for(4 * a->nside, 256), 256, 0, s>>>(a->nside, 0.0, t, true);
    } else {
      ring_table_kernel<<<grid_for(4 * a->nside, 256), 256, 0, s>>>(a->nside, 0.0, t, false);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "built-in ring table kernels");
    k.ring_table = t;
  } else {
    k.ring_table = nullptr;
  }
  return dispatch_types(k, a->interp, has_qu, a->map_dtype, a->params_dtype, s);
}

extern "C" int64_t todgpu_gather_wait_timeouts(void) {
  unsigned long long v = 0;
  if (cudaMemcpyFromSymbol(&v, g_gather_wait_timeouts, sizeof(v)) != cudaSuccess) return -1;
  return (int64_t)v;
}

extern "C" int todgpu_gather_accum_batched(const todgpu_gather_args* jobs, int32_t njobs, int64_t tile,
                                           void* stream) {
  if (njobs < 0) return fail(TODGPU_ESHAPE, "njobs < 0");
  if (njobs == 0) return TODGPU_OK;
  if (!jobs) return fail(TODGPU_EINVAL, "jobs is NULL");
  if (tile < 1 || tile > (1LL << 24)) return fail(TODGPU_ESHAPE, "tile must be in [1, 2^24] samples");
  const todgpu_gather_args& j0 = jobs[0];
  for (int j = 0; j < njobs; ++j) {
    const todgpu_gather_args& a = jobs[j];
    const int rc = check_common(&a, true);
    if (rc != TODGPU_OK) return fail(rc, "job " + std::to_string(j) + ": " + g_last_error);
    if (a.interp != j0.interp || a.nside != j0.nside || a.C != j0.C || a.c_q != j0.c_q || a.c_u != j0.c_u ||
        a.params_dtype != j0.params_dtype || a.map_dtype != j0.map_dtype ||
        (a.flags & TODGPU_FLAG_NO_TABLES) != (j0.flags & TODGPU_FLAG_NO_TABLES))
      return fail(TODGPU_EINVAL, "job " + std::to_string(j) +
                                     ": interp, nside, components, dtypes and flags must match job 0");
  }
  const bool has_qu = j0.c_q >= 0 && j0.c_u >= 0;
  const bool iqu = has_qu && j0.C == 3 && j0.c_q == 1 && j0.c_u == 2;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  static thread_local BatchParams bp;  // ~22 KB: kept off the stack
  for (int first = 0; first < njobs; first += kMaxBatchJobs) {
    const int n = std::min(njobs - first, kMaxBatchJobs);
    bp.njobs = n;
    bp.tile = tile;
    bp.tiles_before[0] = 0;
    bool any_table = false;
    for (int j = 0; j < n; ++j) {
      const todgpu_gather_args& a = jobs[first + j];
      bp.job[j] = make_kargs(&a);
      any_table = any_table || bp.job[j].ring_table != nullptr;
      const long long ntiles = (a.S > 0) ? (a.B + tile - 1) / tile : 0;
      bp.tiles_before[j + 1] = bp.tiles_before[j] + ntiles;
    }
    const int rc = dispatch_batched(bp, j0.interp, has_qu, iqu, any_table, j0.map_dtype, j0.params_dtype, s);
    if (rc != TODGPU_OK) return rc;
  }
  return TODGPU_OK;
}

extern "C" int todgpu_bilinear_stencils(const todgpu_gather_args* a, int64_t* pix, double* wgt, void* stream) {
  int rc = check_common(a, false);
  if (rc != TODGPU_OK) return rc;
  if (a->B == 0 || a->S == 0) return TODGPU_OK;
  if (!pix || !wgt) return fail(TODGPU_EINVAL, "NULL output");
  const KArgs k = make_kargs(a);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int g = grid_for(a->B * a->S, 256);
  if (a->params_dtype == TODGPU_F32)
    stencil_kernel<kParamsRef32><<<g, 256, 0, s>>>(k, reinterpret_cast<long long*>(pix), wgt);
  else if (a->params_dtype == TODGPU_F64)
    stencil_kernel<kParamsF64><<<g, 256, 0, s>>>(k, reinterpret_cast<long long*>(pix), wgt);
  else
    stencil_kernel<kAngles><<<g, 256, 0, s>>>(k, reinterpret_cast<long long*>(pix), wgt);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "stencil_kernel launch");
}

extern "C" int todgpu_get_interp_weights(int64_t nside, const double* theta, const double* phi, int64_t N,
                                         int64_t* pix, double* wgt, void* stream) {
  if (nside < 1 || nside > kMaxNside) return fail(TODGPU_ENSIDE, "nside out of range");
  if (N < 0) return fail(TODGPU_ESHAPE, "N < 0");
  if (N == 0) return TODGPU_OK;
  if (!theta || !phi || !pix || !wgt) return fail(TODGPU_EINVAL, "NULL pointer");
  interp_weights_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nside, theta, phi, N, reinterpret_cast<long long*>(pix), wgt);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "interp_weights_kernel launch");
}

extern "C" int todgpu_ang2pix(int64_t nside, const double* theta, const double* phi, int64_t N, int64_t* pix,
                              void* stream) {
  if (nside < 1 || nside > kMaxNside) return fail(TODGPU_ENSIDE, "nside out of range");
  if (N < 0) return fail(TODGPU_ESHAPE, "N < 0");
  if (N == 0) return TODGPU_OK;
  if (!theta || !phi || !pix) return fail(TODGPU_EINVAL, "NULL pointer");
  ang2pix_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nside, theta, phi, N, reinterpret_cast<long long*>(pix));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "ang2pix_kernel launch");
}

extern "C" int todgpu_pix2ang(int64_t nside, const int64_t* pix, int64_t N, double* theta, double* phi,
                              void* stream) {
  if (nside < 1 || nside > kMaxNside) return fail(TODGPU_ENSIDE, "nside out of range");
  if (N < 0) return fail(TODGPU_ESHAPE, "N < 0");
  if (N == 0) return TODGPU_OK;
  if (!theta || !phi || !pix) return fail(TODGPU_EINVAL, "NULL pointer");
  pix2ang_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nside, reinterpret_cast<const long long*>(pix), N, theta, phi);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "pix2ang_kernel launch");
}

extern "C" int todgpu_spin2(const double* z_pix, const double* sth_pix, const double* phi_pix, const double* z_pts,
                            const double* sth_pts, const double* phi_pts, int64_t N, double* c2d, double* s2d,
                            void* stream) {
  if (N < 0) return fail(TODGPU_ESHAPE, "N < 0");
  if (N == 0) return TODGPU_OK;
  if (!z_pix || !sth_pix || !phi_pix || !z_pts || !sth_pts || !phi_pts || !c2d || !s2d)
    return fail(TODGPU_EINVAL, "NULL pointer");
  spin2_kernel<<<grid_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(z_pix, sth_pix, phi_pix, z_pts,
                                                                                 sth_pts, phi_pts, N, c2d, s2d);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "spin2_kernel launch");
}

extern "C" int todgpu_boresight_phi_host(const float* ax_pts, int64_t B, float* out, int32_t nthreads) {
  if (B < 0) return fail(TODGPU_ESHAPE, "B < 0");
  if (B == 0) return TODGPU_OK;
  if (!ax_pts || !out) return fail(TODGPU_EINVAL, "NULL pointer");
  unsigned hw = std::thread::hardware_concurrency();
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, hw);
  if (B < 65536) nt = 1;
  auto work = [&](int64_t lo, int64_t hi) {
    for (int64_t b = lo; b < hi; ++b) out[b] = atan2f(ax_pts[3 * b + 1], ax_pts[3 * b]);
  };
  if (nt == 1) {
    work(0, B);
    return TODGPU_OK;
  }
  std::vector<std::thread> pool;
  const int64_t step = (B + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const int64_t lo = t * step, hi = std::min<int64_t>(B, lo + step);
    if (lo < hi) pool.emplace_back(work, lo, hi);
  }
  for (auto& th : pool) th.join();
  return TODGPU_OK;
}

extern "C" size_t todgpu_ring_table_bytes(int64_t nside) {
  if (nside < 1 || nside > kMaxNside) return 0;
  return sizeof(RingRec) * (size_t)(4 * nside);
}

extern "C" int todgpu_ring_table_build(int64_t nside, double reach, void* table, size_t bytes, void* stream) {
  if (nside < 1 || nside > kMaxNside) return fail(TODGPU_ENSIDE, "nside out of range");
  if (!table) return fail(TODGPU_EINVAL, "NULL table");
  if (bytes < todgpu_ring_table_bytes(nside)) return fail(TODGPU_ESHAPE, "ring table buffer too small");
  if (((uintptr_t)table & 15) != 0) return fail(TODGPU_EINVAL, "ring table must be 16-byte aligned");
  if (!(reach >= 0.0) || !(reach <= kPi)) return fail(TODGPU_EINVAL, "reach must be in [0, pi]");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  RingRec* t = static_cast<RingRec*>(table);
  ring_table_kernel<<<grid_for(4 * nside, 256), 256, 0, s>>>(nside, reach, t, false);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "ring table kernels");
}

extern "C" int todgpu_fp64_probe(int64_t blocks, int32_t iters, double* sink, double* flops, void* stream) {
  if (blocks < 1 || iters < 1 || !sink || !flops) return fail(TODGPU_EINVAL, "bad probe arguments");
  fp64_probe_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(iters, 0.5, sink);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "fp64_probe_kernel launch");
  *flops = 2.0 * 8.0 * (double)iters * 256.0 * (double)blocks;
  return TODGPU_OK;
}

// Pointing preparation on the device: per sample the float64 rotation
// parameters of tod_rotations.py:306-333 derived from the angles exactly as
// the gather kernel's angles mode derives them (rot_from_angles), written
// structure-of-arrays for the float64-parameter mode.
__global__ void pointing_params_kernel(const KArgs k, double* axes, double* cos_a, double* sin_a, double* pts,
                                       double* cos_p, double* sin_p) {
  for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < k.B;
       b += (long long)gridDim.x * blockDim.x) {
    const SampleRot r = rot_from_angles(k, b);
    axes[3 * b] = r.kx;
    axes[3 * b + 1] = r.ky;
    axes[3 * b + 2] = r.kz;
    cos_a[b] = r.ca;
    sin_a[b] = r.sa;
    pts[3 * b] = r.px;
    pts[3 * b + 1] = r.py;
    pts[3 * b + 2] = r.pz;
    cos_p[b] = r.cp;
    sin_p[b] = r.sp;
  }
}

// L2 bandwidth probe: every thread streams 16-byte loads that bypass L1
// (ld.global.cg) over a buffer that fits in L2, `iters` passes.
__global__ void l2_probe_kernel(const uint4* buf, long long n16, int iters, unsigned* sink) {
  unsigned acc = 0;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (int it = 0; it < iters; ++it)
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n16; i += stride) {
      const uint4 v = __ldcg(buf + i);
      acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
  if (acc == 0x9e3779b9u) sink[blockIdx.x] = acc;  // keeps the loads; practically never true
}

extern "C" int todgpu_pointing_params(const void* theta, const void* phi, const void* psi, int32_t angles_dtype,
                                      int64_t B, double center_phi, double center_theta, double* axes, double* cos_a,
                                      double* sin_a, double* pts, double* cos_p, double* sin_p, void* stream) {
  if (B < 0) return fail(TODGPU_ESHAPE, "B must be >= 0");
  if (B == 0) return TODGPU_OK;
  if (!theta || !phi || !psi || !axes || !cos_a || !sin_a || !pts || !cos_p || !sin_p)
    return fail(TODGPU_EINVAL, "NULL pointer");
  if (angles_dtype != TODGPU_F32 && angles_dtype != TODGPU_F64) return fail(TODGPU_EDTYPE, "bad angles_dtype");
  todgpu_gather_args a{};
  a.B = B;
  a.theta = theta;
  a.phi = phi;
  a.psi = psi;
  a.angles_dtype = angles_dtype;
  a.center_phi = center_phi;
  a.center_theta = center_theta;
  const KArgs k = make_kargs(&a);
  pointing_params_kernel<<<grid_for(B, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(k, axes, cos_a, sin_a, pts,
                                                                                        cos_p, sin_p);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "pointing_params_kernel launch");
}

extern "C" int todgpu_l2_probe(const void* buf, size_t bytes, int32_t iters, unsigned* sink, int64_t blocks,
                               double* bytes_read, void* stream) {
  if (!buf || !sink || !bytes_read || bytes < 16 || iters < 1 || blocks < 1)
    return fail(TODGPU_EINVAL, "bad probe arguments");
  if (((uintptr_t)buf & 15) != 0) return fail(TODGPU_EINVAL, "buffer must be 16-byte aligned");
  const long long n16 = (long long)(bytes / 16);
  l2_probe_kernel<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const uint4*>(buf),
                                                                                   n16, iters, sink);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "l2_probe_kernel launch");
  *bytes_read = 16.0 * (double)n16 * (double)iters;
  return TODGPU_OK;
}

extern "C" int todgpu_pack_map(const void* planar, int32_t planar_dtype, int64_t C, int64_t N, int64_t stride,
                               int32_t packed_dtype, void* out, void* stream) {
  if (!planar || !out) return fail(TODGPU_EINVAL, "NULL pointer");
  if (C < 1 || C > 4 || N < 0 || stride < N) return fail(TODGPU_ESHAPE, "bad map shape");
  if (planar_dtype != TODGPU_F32 && planar_dtype != TODGPU_F64) return fail(TODGPU_EDTYPE, "planar dtype");
  if (packed_dtype != TODGPU_PACKED_F32 && packed_dtype != TODGPU_PACKED_BF16 && packed_dtype != TODGPU_PACKED_F64)
    return fail(TODGPU_EDTYPE, "packed dtype");
  if (((uintptr_t)out & (packed_dtype == TODGPU_PACKED_BF16 ? 7 : 15)) != 0)
    return fail(TODGPU_EINVAL, "packed map must be aligned to 16 bytes (8 for bfloat16 records)");
  if (N == 0) return TODGPU_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int g = grid_for(N, 256);
  if (packed_dtype == TODGPU_PACKED_F64) {
    if (planar_dtype == TODGPU_F32)
      pack_map_f64_kernel<float><<<g, 256, 0, s>>>(static_cast<const float*>(planar), (int)C, N, stride, out);
    else
      pack_map_f64_kernel<double><<<g, 256, 0, s>>>(static_cast<const double*>(planar), (int)C, N, stride, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "pack_map_f64_kernel launch");
  }
  const bool bf = packed_dtype == TODGPU_PACKED_BF16;
  if (planar_dtype == TODGPU_F32) {
    if (bf)
      pack_map_kernel<float, true><<<g, 256, 0, s>>>(static_cast<const float*>(planar), (int)C, N, stride, out);
    else
      pack_map_kernel<float, false><<<g, 256, 0, s>>>(static_cast<const float*>(planar), (int)C, N, stride, out);
  } else {
    if (bf)
      pack_map_kernel<double, true><<<g, 256, 0, s>>>(static_cast<const double*>(planar), (int)C, N, stride, out);
    else
      pack_map_kernel<double, false><<<g, 256, 0, s>>>(static_cast<const double*>(planar), (int)C, N, stride, out);
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, "pack_map_kernel launch");
}

extern "C" int todgpu_abi_version(void) { return TODGPU_ABI_VERSION; }

extern "C" const char* todgpu_last_error_string(void) { return g_last_error.c_str(); }
