// tod_gather.cu -- fused beam-convolution TOD kernels for B200 (sm_100a) and
// the C ABI declared in include/todgpu.h.
//
// Work decomposition: a persistent grid of 256-thread CTAs walks the sample
// batch in tiles of 8 consecutive samples; each warp owns one sample of the
// tile and its 32 lanes stride over the beam pixels, so the per-sample
// rotation scalars are warp-uniform and every lane runs the full per-pixel
// pipeline (rotate -> atan2/clamp -> RING stencil -> spin-2 -> gather ->
// FP64 accumulate).  Lane partial sums are combined with warp shuffles and
// lane 0 adds the result into tod[c, b]; each sample has exactly one writer,
// so no atomics are needed and repeated runs are bit-reproducible.
//
// The beam (unit vectors + weights) is staged in shared memory in chunks of
// kChunk pixels as {vx, vy, vz, w} records; when the whole beam fits it is
// loaded once per CTA and stays resident for every tile.
//
// Compiled with -fmad=false: the pixel decisions and the FP64 accumulation
// reproduce the reference's uncontracted arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "healpix_ring.cuh"
#include "todgpu.h"

namespace todgpu {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kChunkF32 = 4096;  // beam pixels per shared-memory chunk (16 B each)
constexpr int kChunkF64 = 2048;  // (32 B each)
constexpr long long kMaxNside = 16384;

thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

static int cuda_fail(cudaError_t e, const char* what) {
  return fail(TODGPU_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

struct BeamF32 {
  float x, y, z, w;
};
struct BeamF64 {
  double x, y, z;
  float w, pad;
};

struct KArgs {
  long long nside, npix, B, S;
  int C, c_q, c_u;
  const void* vec;
  const void* axes;
  const void* cos_a;
  const void* sin_a;
  const void* pts;
  const void* cos_p;
  const void* sin_p;
  const float* bore_phi;
  const float* beam;
  const void* map;
  long long map_stride;
  double* tod;
  long long tod_stride;
  unsigned long long* err;
};

template <bool P64>
struct ParamTraits;
template <>
struct ParamTraits<false> {
  using Beam = BeamF32;
  static constexpr int kChunk = kChunkF32;
};
template <>
struct ParamTraits<true> {
  using Beam = BeamF64;
  static constexpr int kChunk = kChunkF64;
};

template <bool P64>
__device__ __forceinline__ SampleRot load_rot(const KArgs& a, long long b) {
  SampleRot r;
  if constexpr (P64) {
    const double* ax = static_cast<const double*>(a.axes) + 3 * b;
    const double* pt = static_cast<const double*>(a.pts) + 3 * b;
    r.kx = ax[0];
    r.ky = ax[1];
    r.kz = ax[2];
    r.ca = static_cast<const double*>(a.cos_a)[b];
    r.sa = static_cast<const double*>(a.sin_a)[b];
    r.px = pt[0];
    r.py = pt[1];
    r.pz = pt[2];
    r.cp = static_cast<const double*>(a.cos_p)[b];
    r.sp = static_cast<const double*>(a.sin_p)[b];
  } else {
    const float* ax = static_cast<const float*>(a.axes) + 3 * b;
    const float* pt = static_cast<const float*>(a.pts) + 3 * b;
    r.fkx = ax[0];
    r.fky = ax[1];
    r.fkz = ax[2];
    r.fca = static_cast<const float*>(a.cos_a)[b];
    r.fsa = static_cast<const float*>(a.sin_a)[b];
    r.px = (double)pt[0];
    r.py = (double)pt[1];
    r.pz = (double)pt[2];
    r.cp = (double)static_cast<const float*>(a.cos_p)[b];
    r.sp = (double)static_cast<const float*>(a.sin_p)[b];
  }
  return r;
}

// Boresight (z, sin theta, phi) of the spin-2 angle.  Float32 parameters use
// the reference's typing: sin theta from a float32 square, phi from float32
// atan2 (host libm value when provided).
template <bool P64>
__device__ __forceinline__ void load_boresight(const KArgs& a, long long b, double& z, double& sth,
                                               double& phi) {
  if constexpr (P64) {
    const double* pt = static_cast<const double*>(a.pts) + 3 * b;
    z = clamp1(pt[2]);
    sth = sqrt(max0(1.0 - pt[2] * pt[2]));
    phi = atan2(pt[1], pt[0]);
  } else {
    const float* pt = static_cast<const float*>(a.pts) + 3 * b;
    const float bz = pt[2];
    const float bz2 = bz * bz;
    z = clamp1((double)bz);
    sth = sqrt(max0(1.0 - (double)bz2));
    if (a.bore_phi != nullptr)
      phi = (double)a.bore_phi[b];
    else
      phi = (double)(float)atan2((double)pt[1], (double)pt[0]);
  }
  if (phi < 0.0) phi += kTwoPi;
}

template <bool P64>
__device__ __forceinline__ void stage_beam(const KArgs& a, typename ParamTraits<P64>::Beam* sm,
                                           long long s0, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const long long s = s0 + i;
    if constexpr (P64) {
      const double* v = static_cast<const double*>(a.vec) + 3 * s;
      BeamF64 e;
      e.x = v[0];
      e.y = v[1];
      e.z = v[2];
      e.w = a.beam[s];
      e.pad = 0.f;
      sm[i] = e;
    } else {
      const float* v = static_cast<const float*>(a.vec) + 3 * s;
      sm[i] = BeamF32{v[0], v[1], v[2], a.beam[s]};
    }
  }
}

template <bool P64>
__device__ __forceinline__ void rotate(const SampleRot& r, const typename ParamTraits<P64>::Beam& e,
                                       double& vx, double& vy, double& vz) {
  if constexpr (P64)
    rot_f64(r, e.x, e.y, e.z, vx, vy, vz);
  else
    rot_ref32(r, e.x, e.y, e.z, vx, vy, vz);
}

template <typename MapT>
__device__ __forceinline__ double map_at(const KArgs& a, int c, long long p) {
  return (double)__ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
}

// mp[c, p] * bv with the nearest kernel's typing (tod_nearest.py:146, :158):
// a float32 map element times the float32 weight is a float32 product.
template <typename MapT>
__device__ __forceinline__ double map_x_beam(const KArgs& a, int c, long long p, float bv) {
  const MapT m = __ldg(static_cast<const MapT*>(a.map) + (long long)c * a.map_stride + p);
  if constexpr (sizeof(MapT) == 4)
    return (double)(m * bv);
  else
    return m * (double)bv;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// One pass of a warp over beam pixels [s_begin, s_end) of a chunk held in
// shared memory, accumulating into acc[0..3].
template <int MODE, bool HAS_QU, typename MapT, bool P64>
__device__ __forceinline__ void accumulate_chunk(const KArgs& a, const SampleRot& rot, double z_pts,
                                                 double sth_pts, double phi_pts,
                                                 const typename ParamTraits<P64>::Beam* sm, int n,
                                                 double acc[4], unsigned long long& nerr) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < n; i += 32) {
    const typename ParamTraits<P64>::Beam e = sm[i];
    double vx, vy, vz;
    rotate<P64>(rot, e, vx, vy, vz);
    const float bvf = e.w;
    const double bv = (double)bvf;
    double phi_w = atan2(vy, vx);
    if (phi_w < 0.0) phi_w += kTwoPi;
    if constexpr (MODE == TODGPU_BILINEAR) {
      const double z = clamp1(vz);
      Stencil st;
      hp_stencil(a.nside, z, phi_w, a.npix, st);
      bool ok = true;
#pragma unroll
      for (int k = 0; k < 4; ++k) ok = ok && ((unsigned long long)st.p[k] < (unsigned long long)a.npix);
      if (!ok) {
        ++nerr;
        continue;
      }
      if constexpr (HAS_QU) {
        double c2[4], s2[4], q[4], u[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const double sth_n = sqrt(max0(1.0 - st.zn[k] * st.zn[k]));
          spin2_c2s2(st.zn[k], sth_n, st.phin[k], z_pts, sth_pts, phi_pts, c2[k], s2[k]);
          q[k] = map_at<MapT>(a, a.c_q, st.p[k]);
          u[k] = map_at<MapT>(a, a.c_u, st.p[k]);
        }
        double tq = (st.w[0] * (q[0] * c2[0] + u[0] * s2[0]) + st.w[1] * (q[1] * c2[1] + u[1] * s2[1]) +
                     st.w[2] * (q[2] * c2[2] + u[2] * s2[2]) + st.w[3] * (q[3] * c2[3] + u[3] * s2[3])) *
                    bv;
        double tu = (st.w[0] * (-q[0] * s2[0] + u[0] * c2[0]) + st.w[1] * (-q[1] * s2[1] + u[1] * c2[1]) +
                     st.w[2] * (-q[2] * s2[2] + u[2] * c2[2]) + st.w[3] * (-q[3] * s2[3] + u[3] * c2[3])) *
                    bv;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= a.C) break;
          if (c == a.c_q) {
            acc[c] += tq;
          } else if (c == a.c_u) {
            acc[c] += tu;
          } else {
            acc[c] += (st.w[0] * map_at<MapT>(a, c, st.p[0]) + st.w[1] * map_at<MapT>(a, c, st.p[1]) +
                       st.w[2] * map_at<MapT>(a, c, st.p[2]) + st.w[3] * map_at<MapT>(a, c, st.p[3])) *
                      bv;
          }
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= a.C) break;
          acc[c] += (st.w[0] * map_at<MapT>(a, c, st.p[0]) + st.w[1] * map_at<MapT>(a, c, st.p[1]) +
                     st.w[2] * map_at<MapT>(a, c, st.p[2]) + st.w[3] * map_at<MapT>(a, c, st.p[3])) *
                    bv;
        }
      }
    } else {
      const double sin_th = sqrt(max0(vx * vx + vy * vy));
      const Nearest nb = hp_nearest(a.nside, vz, sin_th, phi_w, a.npix);
      if ((unsigned long long)nb.pix >= (unsigned long long)a.npix) {
        ++nerr;
        continue;
      }
      if constexpr (HAS_QU) {
        const double sth_n = sqrt(max0(1.0 - nb.zc * nb.zc));
        double c2d, s2d;
        spin2_c2s2(nb.zc, sth_n, nb.phic, z_pts, sth_pts, phi_pts, c2d, s2d);
        const double qv = map_at<MapT>(a, a.c_q, nb.pix);
        const double uv = map_at<MapT>(a, a.c_u, nb.pix);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= a.C) break;
          if (c == a.c_q)
            acc[c] += (qv * c2d + uv * s2d) * bv;
          else if (c == a.c_u)
            acc[c] += (-qv * s2d + uv * c2d) * bv;
          else
            acc[c] += map_x_beam<MapT>(a, c, nb.pix, bvf);
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          if (c >= a.C) break;
          acc[c] += map_x_beam<MapT>(a, c, nb.pix, bvf);
        }
      }
    }
  }
}

template <int MODE, bool HAS_QU, typename MapT, bool P64>
__global__ void __launch_bounds__(kThreads) gather_accum_kernel(const KArgs a) {
  using Beam = typename ParamTraits<P64>::Beam;
  constexpr int kChunk = ParamTraits<P64>::kChunk;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Beam* sm = reinterpret_cast<Beam*>(smem_raw);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const long long n_chunks = (a.S + kChunk - 1) / kChunk;
  const bool resident = (n_chunks == 1);
  if (resident) {
    stage_beam<P64>(a, sm, 0, (int)a.S);
    __syncthreads();
  }
  unsigned long long nerr = 0;
  for (long long tile = (long long)blockIdx.x * kWarps; tile < a.B; tile += (long long)gridDim.x * kWarps) {
    const long long b = tile + warp;
    const bool active = (b < a.B);
    SampleRot rot;
    double z_pts = 0.0, sth_pts = 0.0, phi_pts = 0.0;
    if (active) {
      rot = load_rot<P64>(a, b);
      if (HAS_QU) load_boresight<P64>(a, b, z_pts, sth_pts, phi_pts);
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long ch = 0; ch < n_chunks; ++ch) {
      const long long s0 = ch * kChunk;
      const int n = (int)min((long long)kChunk, a.S - s0);
      if (!resident) {
        __syncthreads();
        stage_beam<P64>(a, sm, s0, n);
        __syncthreads();
      }
      if (active) accumulate_chunk<MODE, HAS_QU, MapT, P64>(a, rot, z_pts, sth_pts, phi_pts, sm, n, acc, nerr);
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        if (c >= a.C) break;
        const double v = warp_sum(acc[c]);
        if (lane == 0) a.tod[(long long)c * a.tod_stride + b] += v;
      }
    }
  }
  if (a.err != nullptr) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nerr += __shfl_xor_sync(0xffffffffu, nerr, o);
    if (lane == 0 && nerr) atomicAdd(a.err, nerr);
  }
}

// ---------------------------------------------------------------------------
// Small parity kernels (one thread per element).
// ---------------------------------------------------------------------------

template <bool P64>
__global__ void stencil_kernel(const KArgs a, long long* pix, double* wgt) {
  const long long BS = a.B * a.S;
  for (long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < BS;
       n += (long long)gridDim.x * blockDim.x) {
    const long long b = n / a.S, s = n - b * a.S;
    const SampleRot rot = load_rot<P64>(a, b);
    double vx, vy, vz;
    if constexpr (P64) {
      const double* v = static_cast<const double*>(a.vec) + 3 * s;
      rot_f64(rot, v[0], v[1], v[2], vx, vy, vz);
    } else {
      const float* v = static_cast<const float*>(a.vec) + 3 * s;
      rot_ref32(rot, v[0], v[1], v[2], vx, vy, vz);
    }
    const double z = clamp1(vz);
    double phi_w = atan2(vy, vx);
    if (phi_w < 0.0) phi_w += kTwoPi;
    Stencil st;
    hp_stencil(a.nside, z, phi_w, a.npix, st);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      pix[k * BS + n] = st.p[k];
      wgt[k * BS + n] = st.w[k];
    }
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
    out[i] = hp_nearest(nside, z, sin(theta[i]), phi_w, npix).pix;
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
// Host side.
// ---------------------------------------------------------------------------

static int sm_count() {
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
  bool configured = false;
};

template <int MODE, bool HAS_QU, typename MapT, bool P64>
static int launch_gather(const KArgs& k, cudaStream_t stream) {
  using Beam = typename ParamTraits<P64>::Beam;
  constexpr int kChunk = ParamTraits<P64>::kChunk;
  auto kern = gather_accum_kernel<MODE, HAS_QU, MapT, P64>;
  static LaunchInfo info;
  static std::mutex mu;
  const size_t smem_max = sizeof(Beam) * kChunk;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (!info.configured) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
      int nb = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, kThreads, smem_max);
      if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
      info.blocks_per_sm = std::max(nb, 1);
      info.configured = true;
    }
  }
  const long long tiles = (k.B + kWarps - 1) / kWarps;
  const long long max_blocks = (long long)sm_count() * info.blocks_per_sm;
  const int grid = (int)std::max(1LL, std::min(tiles, max_blocks));
  const size_t smem = sizeof(Beam) * (size_t)std::min<long long>(k.S, kChunk);
  kern<<<grid, kThreads, smem, stream>>>(k);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "gather_accum_kernel launch");
  return TODGPU_OK;
}

template <int MODE, typename MapT, bool P64>
static int dispatch_qu(const KArgs& k, bool has_qu, cudaStream_t s) {
  return has_qu ? launch_gather<MODE, true, MapT, P64>(k, s) : launch_gather<MODE, false, MapT, P64>(k, s);
}

template <int MODE>
static int dispatch_types(const KArgs& k, bool has_qu, int map_dtype, int params_dtype, cudaStream_t s) {
  if (map_dtype == TODGPU_F32) {
    return params_dtype == TODGPU_F32 ? dispatch_qu<MODE, float, false>(k, has_qu, s)
                                      : dispatch_qu<MODE, float, true>(k, has_qu, s);
  }
  return params_dtype == TODGPU_F32 ? dispatch_qu<MODE, double, false>(k, has_qu, s)
                                    : dispatch_qu<MODE, double, true>(k, has_qu, s);
}

static int check_common(const todgpu_gather_args* a, bool need_map) {
  if (a == nullptr) return fail(TODGPU_EINVAL, "args is NULL");
  if (a->abi_version != TODGPU_ABI_VERSION)
    return fail(TODGPU_EABI, "abi_version " + std::to_string(a->abi_version) + " != " +
                                 std::to_string(TODGPU_ABI_VERSION));
  if (a->nside < 1 || a->nside > kMaxNside)
    return fail(TODGPU_ENSIDE, "nside " + std::to_string(a->nside) + " outside [1, 16384]");
  if (a->B < 0 || a->S < 0) return fail(TODGPU_ESHAPE, "negative B or S");
  if (a->params_dtype != TODGPU_F32 && a->params_dtype != TODGPU_F64)
    return fail(TODGPU_EDTYPE, "params_dtype must be TODGPU_F32 or TODGPU_F64");
  if (a->B > 0 && a->S > 0) {
    if (!a->vec_orig || !a->axes || !a->cos_a || !a->sin_a || !a->ax_pts || !a->cos_p || !a->sin_p)
      return fail(TODGPU_EINVAL, "NULL parameter array");
  }
  if (need_map) {
    if (a->interp != TODGPU_BILINEAR && a->interp != TODGPU_NEAREST)
      return fail(TODGPU_EINVAL, "interp must be TODGPU_BILINEAR or TODGPU_NEAREST");
    if (a->C < 1 || a->C > 4) return fail(TODGPU_ESHAPE, "C must be in [1, 4]");
    if (a->c_q < -1 || a->c_q >= a->C || a->c_u < -1 || a->c_u >= a->C)
      return fail(TODGPU_ESHAPE, "c_q/c_u must be -1 or a component index");
    if (a->c_q >= 0 && a->c_q == a->c_u) return fail(TODGPU_ESHAPE, "c_q == c_u");
    if (a->map_dtype != TODGPU_F32 && a->map_dtype != TODGPU_F64)
      return fail(TODGPU_EDTYPE, "map_dtype must be TODGPU_F32 or TODGPU_F64");
    const long long npix = 12 * a->nside * a->nside;
    if (a->map_stride < npix) return fail(TODGPU_ESHAPE, "map_stride < 12*nside^2");
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
  k.beam = a->beam_vals;
  k.map = a->map;
  k.map_stride = a->map_stride;
  k.tod = a->tod;
  k.tod_stride = a->tod_stride;
  k.err = a->err_count;
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
  if (a->interp == TODGPU_BILINEAR) return dispatch_types<TODGPU_BILINEAR>(k, has_qu, a->map_dtype, a->params_dtype, s);
  return dispatch_types<TODGPU_NEAREST>(k, has_qu, a->map_dtype, a->params_dtype, s);
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
    stencil_kernel<false><<<g, 256, 0, s>>>(k, reinterpret_cast<long long*>(pix), wgt);
  else
    stencil_kernel<true><<<g, 256, 0, s>>>(k, reinterpret_cast<long long*>(pix), wgt);
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

extern "C" int todgpu_abi_version(void) { return TODGPU_ABI_VERSION; }

extern "C" const char* todgpu_last_error_string(void) { return g_last_error.c_str(); }
