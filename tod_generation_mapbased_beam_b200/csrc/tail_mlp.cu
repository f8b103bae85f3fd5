// tail_mlp.cu -- the learned far-sidelobe tail: a Fourier-feature MLP of the
// pointing (boresight unit vector and roll psi) that predicts the I/Q/U TOD
// contribution of a beam's far sidelobes, trained and evaluated on the GPU by
// the kernels in this file.
//
// Network (row-major weights, one flat parameter vector):
//   x     = (sin t cos p, sin t sin p, cos t, cos psi, sin psi, cos 2psi, sin 2psi)
//   f     = [cos(2 pi B x), sin(2 pi B x)]            B: (F, 7) fixed, 2F features
//   a_1   = silu(W_0 f + b_0)                         W_0: (H, 2F)
//   a_l+1 = silu(W_l a_l + b_l), l = 1 .. D-1         W_l: (H, H)
//   y     = W_D a_D + b_D                             W_D: (O, H)
// Weights are used in bfloat16 (a copy of the float32 master parameters that
// the Adam step refreshes), activations are stored in bfloat16 and every
// contraction accumulates in float32: the hidden layers on the tensor cores --
// forward products on tcgen05 with TMEM accumulators and TMA-staged operands
// (widths 128 and 256), backward products and other widths on mma.sync
// m16n8k16 bf16 -> f32 -- the O <= 4 wide head on the CUDA cores.  Pre-activations are kept in float32 for
// the backward pass.  Weight gradients over the batch use a fixed split of
// the batch and a fixed-order reduction, so training is deterministic.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>

#include "gather_impl.cuh"

namespace todgpu {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int kIn = 7;
constexpr int kMaxDepth = 8;
constexpr int kMaxOut = 4;
constexpr int BM = 128, BN = 128, BK = 32;
constexpr int kLd = BK + 8;  // shared-memory row stride in elements (80 B: conflict-free ldmatrix)
constexpr int kThreads = 256;

struct Dims {
  int F, H, D, O;
  int K(int l) const { return l == 0 ? 2 * F : H; }  // input width of hidden layer l
};

struct Offsets {
  long long w[kMaxDepth + 1], b[kMaxDepth + 1];  // hidden layers 0..D-1, head at D
  long long total;
};

inline Offsets param_offsets(const Dims& d) {
  Offsets o{};
  long long p = 0;
  for (int l = 0; l < d.D; ++l) {
    o.w[l] = p;
    p += (long long)d.H * d.K(l);
    o.b[l] = p;
    p += d.H;
  }
  o.w[d.D] = p;
  p += (long long)d.O * d.H;
  o.b[d.D] = p;
  p += d.O;
  o.total = p;
  return o;
}

// Workspace regions for a batch of M rows (byte offsets, 256-B aligned).
enum Region { R_X, R_FEAT, R_Z, R_A, R_Y, R_DZ, R_PART, R_LOSS, R_COUNT };

inline int splits_for(long long M) {
  int s = 1;
  while (s < 64 && M % ((long long)s * 2 * BM) == 0 && M / (s * 2) >= 256) s *= 2;
  return s;
}

inline long long part_floats(const Dims& d, long long M) {
  const long long s = splits_for(M);
  const long long gemm = s * d.H * std::max(2LL * d.F, (long long)d.H);
  const long long head = s * ((long long)d.O * d.H + d.O);
  const long long bias = s * d.H;
  return std::max(gemm, std::max(head, bias));
}

inline void ws_offsets(const Dims& d, long long M, long long* off) {
  auto al = [](long long x) { return (x + 255) / 256 * 256; };
  long long p = 0;
  off[R_X] = p;
  p = al(p + M * kIn * 4);
  off[R_FEAT] = p;
  p = al(p + M * 2LL * d.F * 2);
  off[R_Z] = p;
  p = al(p + (long long)d.D * M * d.H * 4);
  off[R_A] = p;
  p = al(p + (long long)d.D * M * d.H * 2);
  off[R_Y] = p;
  p = al(p + M * d.O * 4);
  off[R_DZ] = p;
  p = al(p + 2LL * M * d.H * 2);
  off[R_PART] = p;
  p = al(p + part_floats(d, M) * 4);
  off[R_LOSS] = p;
  p = al(p + (M + 1) * 4);
  off[R_COUNT] = p;
}

// ---------------------------------------------------------------------------
// inputs and Fourier features
// ---------------------------------------------------------------------------
template <typename T>
__global__ void inputs_kernel(const T* theta, const T* phi, const T* psi, long long n, long long M, float* x) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M; i += (long long)gridDim.x * blockDim.x) {
    float* o = x + i * kIn;
    if (i >= n) {
      for (int k = 0; k < kIn; ++k) o[k] = 0.0f;
      continue;
    }
    double st, ct, sp, cp, ss, cs;
    sincos((double)theta[i], &st, &ct);
    sincos((double)phi[i], &sp, &cp);
    sincos((double)psi[i], &ss, &cs);
    o[0] = (float)(st * cp);
    o[1] = (float)(st * sp);
    o[2] = (float)ct;
    o[3] = (float)cs;
    o[4] = (float)ss;
    o[5] = (float)(cs * cs - ss * ss);
    o[6] = (float)(2.0 * ss * cs);
  }
}

__global__ void features_kernel(const float* x, long long M, const float* freq, int F, bf16* feat) {
  const long long total = M * F;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long m = t / F;
    const int j = (int)(t - m * F);
    const float* xm = x + m * kIn;
    const float* bj = freq + (long long)j * kIn;
    float z = 0.0f;
    for (int k = 0; k < kIn; ++k) z += bj[k] * xm[k];
    float s, c;
    sincospif(2.0f * z, &s, &c);  // (sin, cos)(2 pi z)
    feat[m * 2 * F + j] = __float2bfloat16(c);
    feat[m * 2 * F + F + j] = __float2bfloat16(s);
  }
}

// ---------------------------------------------------------------------------
// tensor-core GEMM: C(m, n) = sum_k A(m, k) B(n, k), bf16 operands, f32 sums
//   AL = 0: A(m, k) = A[m * lda + k]      AL = 1: A(m, k) = A[k * lda + m]
//   BL = 0: B(n, k) = B[n * ldb + k]      BL = 1: B(n, k) = B[k * ldb + n]
// CTA tile 128 x 128 x 32, 8 warps as 2 (m) x 4 (n), warp tile 64 x 32.
// blockIdx.z selects a contiguous range of K (split-K partial sums).
// M, N multiples of 128 and K a multiple of 32 (checked on the host).
// ---------------------------------------------------------------------------
enum Epi { EPI_FWD = 0, EPI_BWD = 1, EPI_PART = 2 };

struct GemmArgs {
  const bf16* A;
  long long lda;
  const bf16* B;
  long long ldb;
  int M, N, K;          // K per split
  const float* bias;    // EPI_FWD: (N,)
  float* zout;          // EPI_FWD: pre-activation (M, ldc) f32, optional
  bf16* aout;           // EPI_FWD: silu(z); EPI_BWD: dz (M, ldc) bf16
  long long ldc;
  const float* zin;     // EPI_BWD: pre-activation of the output columns (M, ldc)
  float* cout;          // EPI_PART: (splits, M, ldc) f32
};

__device__ __forceinline__ float silu_f(float v) { return v / (1.0f + expf(-v)); }
__device__ __forceinline__ float dsilu_f(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned& r0, unsigned& r1, unsigned& r2, unsigned& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float* c, const unsigned* a, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Global -> registers: the 128 x 32 tile of one operand as two 16-byte chunks per thread.
template <int L>
__device__ __forceinline__ void load_tile(const bf16* P, long long ld, int r0, long long k0, uint4* reg) {
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int c = threadIdx.x + i * kThreads;
    if (L == 0) {  // row r, 8 consecutive k
      const int r = c >> 2, kc = (c & 3) * 8;
      reg[i] = *reinterpret_cast<const uint4*>(P + (long long)(r0 + r) * ld + k0 + kc);
    } else {  // k row kr, 8 consecutive rows
      const int kr = c >> 4, rc = (c & 15) * 8;
      reg[i] = *reinterpret_cast<const uint4*>(P + (k0 + kr) * ld + r0 + rc);
    }
  }
}

// Registers -> shared tile S[row][k] (k contiguous, row stride kLd).
template <int L>
__device__ __forceinline__ void store_tile(bf16* S, const uint4* reg) {
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int c = threadIdx.x + i * kThreads;
    if (L == 0) {
      const int r = c >> 2, kc = (c & 3) * 8;
      *reinterpret_cast<uint4*>(S + r * kLd + kc) = reg[i];
    } else {
      const int kr = c >> 4, rc = (c & 15) * 8;
      const bf16* v = reinterpret_cast<const bf16*>(&reg[i]);
#pragma unroll
      for (int j = 0; j < 8; ++j) S[(rc + j) * kLd + kr] = v[j];
    }
  }
}

template <int AL, int BL, int EPI>
__global__ void __launch_bounds__(kThreads) gemm_kernel(GemmArgs g) {
  __shared__ __align__(16) bf16 As[BM * kLd];
  __shared__ __align__(16) bf16 Bs[BN * kLd];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const long long kb = (long long)blockIdx.z * g.K;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.0f;

  uint4 ra[2], rb[2];
  load_tile<AL>(g.A, g.lda, m0, kb, ra);
  load_tile<BL>(g.B, g.ldb, n0, kb, rb);
  const unsigned sA = (unsigned)__cvta_generic_to_shared(As);
  const unsigned sB = (unsigned)__cvta_generic_to_shared(Bs);

  for (int kt = 0; kt < g.K; kt += BK) {
    __syncthreads();  // the previous tile is no longer read
    store_tile<AL>(As, ra);
    store_tile<BL>(Bs, rb);
    __syncthreads();
    if (kt + BK < g.K) {  // prefetch the next tile while this one is multiplied
      load_tile<AL>(g.A, g.lda, m0, kb + kt + BK, ra);
      load_tile<BL>(g.B, g.ldb, n0, kb + kt + BK, rb);
    }
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      unsigned af[4][4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        const int row = wm + mt * 16 + (lane & 15);
        const int col = ks + (lane >> 4) * 8;
        ldsm_x4(sA + (unsigned)(row * kLd + col) * 2u, af[mt][0], af[mt][1], af[mt][2], af[mt][3]);
      }
      unsigned bfr[4][2];
#pragma unroll
      for (int np = 0; np < 2; ++np) {
        const int row = wn + np * 16 + (lane & 7) + ((lane >> 4) << 3);
        const int col = ks + ((lane >> 3) & 1) * 8;
        ldsm_x4(sB + (unsigned)(row * kLd + col) * 2u, bfr[2 * np][0], bfr[2 * np][1], bfr[2 * np + 1][0],
                bfr[2 * np + 1][1]);
      }
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], af[mt], bfr[nt][0], bfr[nt][1]);
    }
  }

  // epilogue: thread holds (row, col..col+1) and (row + 8, col..col+1) of each 16 x 8 tile
#pragma unroll
  for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      const int col = n0 + wn + nt * 8 + (lane & 3) * 2;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int row = m0 + wm + mt * 16 + (lane >> 2) + h * 8;
        float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
        const long long o = (long long)row * g.ldc + col;
        if (EPI == EPI_FWD) {
          v0 += g.bias[col];
          v1 += g.bias[col + 1];
          if (g.zout) *reinterpret_cast<float2*>(g.zout + o) = make_float2(v0, v1);
          *reinterpret_cast<__nv_bfloat162*>(g.aout + o) = __floats2bfloat162_rn(silu_f(v0), silu_f(v1));
        } else if (EPI == EPI_BWD) {
          const float2 z = *reinterpret_cast<const float2*>(g.zin + o);
          *reinterpret_cast<__nv_bfloat162*>(g.aout + o) =
              __floats2bfloat162_rn(v0 * dsilu_f(z.x), v1 * dsilu_f(z.y));
        } else {
          float* c = g.cout + (long long)blockIdx.z * g.M * g.ldc;
          *reinterpret_cast<float2*>(c + o) = make_float2(v0, v1);
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// head (O <= 4 outputs, CUDA cores), loss, and their gradients
// ---------------------------------------------------------------------------
struct HeadOut {
  // training: target (M, O) normalised, dy (M, O), loss (M,) squared error per row
  const float* target;
  float* dy;
  float* loss;
  float grad_scale;  // d(mean loss)/d(residual) = 2 / (M O)
  // inference: tod[rows[o] * tod_stride + b0 + m] += y_o * scale[o] + shift[o] for m < n_valid
  double* tod;
  long long tod_stride, b0, n_valid;
  int rows[kMaxOut];
  double scale[kMaxOut], shift[kMaxOut];
  // plain forward: y (M, O)
  float* y;
};

template <int O>
__global__ void head_kernel(const bf16* act, long long M, int H, const bf16* Wo, const float* bo, HeadOut h) {
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long m = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); m < M; m += warps) {
    float s[O];
#pragma unroll
    for (int o = 0; o < O; ++o) s[o] = 0.0f;
    for (int k = lane * 8; k < H; k += 256) {
      const uint4 av = *reinterpret_cast<const uint4*>(act + m * H + k);
      const bf16* a8 = reinterpret_cast<const bf16*>(&av);
#pragma unroll
      for (int o = 0; o < O; ++o) {
        const uint4 wv = *reinterpret_cast<const uint4*>(Wo + (long long)o * H + k);
        const bf16* w8 = reinterpret_cast<const bf16*>(&wv);
#pragma unroll
        for (int j = 0; j < 8; ++j) s[o] += __bfloat162float(a8[j]) * __bfloat162float(w8[j]);
      }
    }
#pragma unroll
    for (int o = 0; o < O; ++o)
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) s[o] += __shfl_xor_sync(0xffffffffu, s[o], d);
    if (lane == 0) {
      float l2 = 0.0f;
#pragma unroll
      for (int o = 0; o < O; ++o) {
        const float y = s[o] + bo[o];
        if (h.target) {
          const float r = y - h.target[m * O + o];
          h.dy[m * O + o] = r * h.grad_scale;
          l2 += r * r;
        }
        if (h.y) h.y[m * O + o] = y;
        if (h.tod && m < h.n_valid) h.tod[h.rows[o] * h.tod_stride + h.b0 + m] += (double)y * h.scale[o] + h.shift[o];
      }
      if (h.loss) h.loss[m] = l2;
    }
  }
}

// dz(m, k) = (sum_o dy(m, o) Wo(o, k)) silu'(z(m, k))
template <int O>
__global__ void head_bwd_kernel(const float* dy, long long M, int H, const bf16* Wo, const float* z, bf16* dz) {
  const long long total = M * H;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long m = t / H;
    const int k = (int)(t - m * H);
    float g = 0.0f;
#pragma unroll
    for (int o = 0; o < O; ++o) g += dy[m * O + o] * __bfloat162float(Wo[(long long)o * H + k]);
    dz[t] = __float2bfloat16(g * dsilu_f(z[t]));
  }
}

// Head weight/bias gradient partials over a contiguous range of rows per block:
// part[z][o * H + k] = sum_m dy(m, o) act(m, k), part[z][O * H + o] = sum_m dy(m, o).
template <int O>
__global__ void head_wgrad_kernel(const float* dy, const bf16* act, long long rows_per_split, int H, float* part) {
  const long long r0 = (long long)blockIdx.x * rows_per_split;
  float* p = part + (long long)blockIdx.x * (O * H + O);
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    float s[O];
#pragma unroll
    for (int o = 0; o < O; ++o) s[o] = 0.0f;
    for (long long m = r0; m < r0 + rows_per_split; ++m) {
      const float a = __bfloat162float(act[m * H + k]);
#pragma unroll
      for (int o = 0; o < O; ++o) s[o] += dy[m * O + o] * a;
    }
#pragma unroll
    for (int o = 0; o < O; ++o) p[o * H + k] = s[o];
  }
  if (threadIdx.x < O) {
    float s = 0.0f;
    for (long long m = r0; m < r0 + rows_per_split; ++m) s += dy[m * O + threadIdx.x];
    p[O * H + threadIdx.x] = s;
  }
}

// Bias gradient partials of a hidden layer: part[z][n] = sum over the split's rows of dz(m, n).
__global__ void colsum_kernel(const bf16* dz, long long rows_per_split, int H, float* part) {
  const long long r0 = (long long)blockIdx.x * rows_per_split;
  for (int n = threadIdx.x; n < H; n += blockDim.x) {
    float s = 0.0f;
    for (long long m = r0; m < r0 + rows_per_split; ++m) s += __bfloat162float(dz[m * H + n]);
    part[(long long)blockIdx.x * H + n] = s;
  }
}

// out[i] = sum_z part[z * count + i], z in increasing order.
__global__ void reduce_splits_kernel(const float* part, int splits, long long count, float* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(long long)z * count + i];
    out[i] = s;
  }
}

// Mean of loss[0..M) into *out (one block, fixed order).
__global__ void loss_mean_kernel(const float* loss, long long M, float inv_count, float* out) {
  __shared__ float red[kThreads];
  float s = 0.0f;
  for (long long i = threadIdx.x; i < M; i += blockDim.x) s += loss[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int d = blockDim.x / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) red[threadIdx.x] += red[threadIdx.x + d];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0] * inv_count;
}

__global__ void adam_kernel(float* p, bf16* pb, float* mo, float* ve, const float* g, long long n, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float m = b1 * mo[i] + (1.0f - b1) * gi;
    const float v = b2 * ve[i] + (1.0f - b2) * gi * gi;
    mo[i] = m;
    ve[i] = v;
    const float q = p[i] - lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    p[i] = q;
    pb[i] = __float2bfloat16(q);
  }
}

__global__ void to_bf16_kernel(const float* p, bf16* pb, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    pb[i] = __float2bfloat16(p[i]);
}

// ---------------------------------------------------------------------------
// Forward layer on the 5th-generation tensor cores (tcgen05, sm_100a), with
// its operands staged by the tensor memory accelerator (TMA):
//   out(m, n) = silu(sum_k A(m, k) W(n, k) + bias(n)),  A (M, K), W (N, K)
//   bf16 row-major; the sums accumulate in float32 in tensor memory (TMEM).
// One CTA of 256 threads per 128-row tile, all N (128 or 256) columns at once
// in N TMEM columns.  K advances in k-tiles of 32 through a ring of 4 shared-
// memory stages.  Lane 0 of warp 0 is the producer and the MMA issuer: it
// starts the TMA copies of a k-tile (A: 128 x 32, W: N x 32) on the stage's
// "full" barrier (transaction count = the stage's bytes), waits for them,
// issues the k-tile's two 128 x N x 16 MMAs and commits them to the stage's
// "empty" barrier, and refills the stage of the previous k-tile once that
// barrier shows its MMAs done.  The tensor maps view each operand as
// (8 elements, rows, K / 8) with strides (2 B, K * 2 B, 16 B), so a box of
// (8, rows, 4) lands in shared memory in the canonical no-swizzle K-major
// layout: 8-row x 16-byte core matrices, 8-row groups 128 B apart, 16-byte K
// chunks one column of row groups apart.  Epilogue: warp w reads TMEM lanes
// 32 (w % 4) .. +31 (its rows) and half of the columns, adds the bias, applies
// SiLU, stores bfloat16 (and the float32 pre-activation when asked).  Every
// wait is bounded; a wait that runs out is counted in g_tc_timeouts and the
// CTA skips the rest of its work, still freeing its TMEM.
// ---------------------------------------------------------------------------
constexpr int TC_BM = 128, TC_BK = 32, TC_STAGES = 4, TC_THREADS = 256;
constexpr int kTcWaitLimit = 1 << 20;
__device__ unsigned int g_tc_timeouts;

template <int N>
struct TcShape {
  static constexpr int A_BYTES = TC_BM * TC_BK * 2;      // 8 KB
  static constexpr int B_BYTES = N * TC_BK * 2;          // 8 or 16 KB
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int SMEM = TC_STAGES * STAGE;
  static constexpr int A_LBO = (TC_BM / 8) * 128;        // byte stride between K chunks
  static constexpr int B_LBO = (N / 8) * 128;
  // instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16
  // (bits 7-9, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24
  static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
                                    ((uint32_t)(TC_BM >> 4) << 24);
};

// shared-memory matrix descriptor: start >> 4 (bits 0-13), leading byte offset
// >> 4 (bits 16-29), stride byte offset >> 4 (bits 32-45), version 1 (bit 46),
// no swizzle (bits 61-63 = 0)
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  for (int it = 0; it < kTcWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMA copies of k-tile kt (A rows m0.., all N rows of W) into stage st.
template <int N>
__device__ __forceinline__ void tc_produce(const CUtensorMap* ta, const CUtensorMap* tw, long long m0, int kt,
                                           uint32_t stage_addr, uint32_t full_bar) {
  using Sh = TcShape<N>;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"((uint32_t)Sh::STAGE), "r"(full_bar)
               : "memory");
  const int kc = kt * (TC_BK / 8);
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(stage_addr),
      "l"(reinterpret_cast<uint64_t>(ta)), "r"(full_bar), "r"(0), "r"((int)m0), "r"(kc)
      : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];" ::
          "r"(stage_addr + (uint32_t)Sh::A_BYTES),
      "l"(reinterpret_cast<uint64_t>(tw)), "r"(full_bar), "r"(0), "r"(0), "r"(kc)
      : "memory");
}

template <int N>
__global__ void __launch_bounds__(TC_THREADS) gemm_tc_fwd_kernel(const __grid_constant__ CUtensorMap tma_a,
                                                                 const __grid_constant__ CUtensorMap tma_w, int K,
                                                                 const float* bias, float* zout, bf16* aout,
                                                                 long long ldc) {
  using Sh = TcShape<N>;
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) unsigned long long bars[2 * TC_STAGES + 1];  // full[S], empty[S], done
  __shared__ uint32_t tmem_slot;
  __shared__ int s_ok;
  __shared__ float s_bias[N];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.x * TC_BM;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(tc_smem);
  const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(bars);
  const uint32_t full0 = bar0, empty0 = bar0 + 8 * TC_STAGES, done = bar0 + 16 * TC_STAGES;
  for (int i = tid; i < N; i += TC_THREADS) s_bias[i] = bias[i];
  if (tid == 0) {
    for (int i = 0; i < 2 * TC_STAGES + 1; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar0 + 8 * i));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    s_ok = 1;
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(&tmem_slot)),
                 "r"(N));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      const int KT = K / TC_BK;
      bool ok = true;
      int produced = 0, consumed = 0;  // k-tiles whose copies were started / waited for
      for (int kt = 0; kt < TC_STAGES && kt < KT; ++kt, ++produced)
        tc_produce<N>(&tma_a, &tma_w, m0, kt, sbase + kt * Sh::STAGE, full0 + 8 * kt);
      for (int kt = 0; kt < KT && ok; ++kt) {
        const int st = kt % TC_STAGES;
        const uint32_t sa = sbase + st * Sh::STAGE, sb = sa + Sh::A_BYTES;
        if (!tc_wait(full0 + 8 * st, (uint32_t)((kt / TC_STAGES) & 1))) {
          ok = false;
          break;
        }
        consumed = kt + 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int s = 0; s < TC_BK / 16; ++s) {
          const uint64_t da = tc_desc(sa + s * 2 * Sh::A_LBO, Sh::A_LBO, 128);
          const uint64_t db = tc_desc(sb + s * 2 * Sh::B_LBO, Sh::B_LBO, 128);
          const uint32_t accumulate = (kt > 0 || s > 0) ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
              "l"(da), "l"(db), "r"(Sh::IDESC), "r"(accumulate));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         empty0 + 8 * st)
                     : "memory");
        // refill the previous k-tile's stage once its MMAs are done
        const int kp = kt - 1, kr = kp + TC_STAGES;
        if (kp >= 0 && kr < KT) {
          const int sp = kp % TC_STAGES;
          if (!tc_wait(empty0 + 8 * sp, (uint32_t)((kp / TC_STAGES) & 1))) {
            ok = false;
            break;
          }
          tc_produce<N>(&tma_a, &tma_w, m0, kr, sbase + sp * Sh::STAGE, full0 + 8 * sp);
          ++produced;
        }
      }
      // after a timeout: let copies already started land before the CTA leaves
      for (int t = consumed; !ok && t < produced; ++t)
        tc_wait(full0 + 8 * (t % TC_STAGES), (uint32_t)((t / TC_STAGES) & 1));
      if (ok) {
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(done)
                     : "memory");
        ok = tc_wait(done, 0);
      }
      if (!ok) {
        s_ok = 0;
        atomicAdd(&g_tc_timeouts, 1u);
      }
    }
    __syncwarp();
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (s_ok) {
    const int q = warp & 3, half = warp >> 2;
    const long long row = m0 + q * 32 + lane;
#pragma unroll 1
    for (int c0 = half * (N / 2); c0 < (half + 1) * (N / 2); c0 += 32) {
      uint32_t r[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
            "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
            "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
            "=r"(r[30]), "=r"(r[31])
          : "r"(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]) + s_bias[c0 + j];
      if (zout) {
        float4* zp = reinterpret_cast<float4*>(zout + row * ldc + c0);
#pragma unroll
        for (int j = 0; j < 8; ++j) zp[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      }
      uint4* ap = reinterpret_cast<uint4*>(aout + row * ldc + c0);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        __nv_bfloat162 h[4];
#pragma unroll
        for (int t = 0; t < 4; ++t)
          h[t] = __floats2bfloat162_rn(silu_f(v[8 * j + 2 * t]), silu_f(v[8 * j + 2 * t + 1]));
        ap[j] = *reinterpret_cast<const uint4*>(h);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(N));
}

// ---------------------------------------------------------------------------
// host orchestration
// ---------------------------------------------------------------------------
inline unsigned grid1d(long long n, int threads) {
  return (unsigned)std::max(1LL, std::min((n + threads - 1) / threads, 148LL * 16));
}

template <int AL, int BL, int EPI>
void gemm(const GemmArgs& g, int splits, cudaStream_t s) {
  dim3 grid(g.N / BN, g.M / BM, splits);
  gemm_kernel<AL, BL, EPI><<<grid, kThreads, 0, s>>>(g);
}

struct Net {
  Dims d;
  Offsets off;
  const float* freq;
  float* p;
  bf16* pb;
  float* grad;
  float* am;
  float* av;
};

struct Ws {
  float* x;
  bf16* feat;
  float* z;
  bf16* a;
  float* y;
  bf16* dz;
  float* part;
  float* loss;
};

inline Ws ws_view(const Dims& d, long long M, void* base) {
  long long o[R_COUNT + 1];
  ws_offsets(d, M, o);
  char* b = static_cast<char*>(base);
  return Ws{reinterpret_cast<float*>(b + o[R_X]),    reinterpret_cast<bf16*>(b + o[R_FEAT]),
            reinterpret_cast<float*>(b + o[R_Z]),    reinterpret_cast<bf16*>(b + o[R_A]),
            reinterpret_cast<float*>(b + o[R_Y]),    reinterpret_cast<bf16*>(b + o[R_DZ]),
            reinterpret_cast<float*>(b + o[R_PART]), reinterpret_cast<float*>(b + o[R_LOSS])};
}

// features of w.x, then the hidden layers (pre-activations kept when keep_z).
// Forward path of the hidden layers: tcgen05 (default) for widths 128 and 256,
// mma.sync otherwise or when selected by todgpu_mlp_set_forward_path.
inline std::atomic<int>& forward_path() {
  static std::atomic<int> path{TODGPU_MLP_TCGEN05};
  return path;
}

inline std::atomic<long long>& tc_launch_count() {
  static std::atomic<long long> n{0};
  return n;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no libcuda link).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// (8 elements, rows, K / 8) view of a row-major (rows, K) bf16 matrix, box (8, box_rows, TC_BK / 8).
inline bool encode_operand(CUtensorMap* map, const bf16* base, long long rows, int K, int box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc) return false;
  const cuuint64_t dims[3] = {8, (cuuint64_t)rows, (cuuint64_t)(K / 8)};
  const cuuint64_t strides[2] = {(cuuint64_t)K * 2, 16};
  const cuuint32_t box[3] = {8, (cuuint32_t)box_rows, TC_BK / 8};
  const cuuint32_t estr[3] = {1, 1, 1};
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int N>
bool launch_tc(const GemmArgs& g, cudaStream_t s) {
  static std::once_flag once;
  static cudaError_t attr = cudaSuccess;
  std::call_once(once, [] {
    attr = cudaFuncSetAttribute(gemm_tc_fwd_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                TcShape<N>::SMEM);
  });
  if (attr != cudaSuccess) return false;
  CUtensorMap ta, tw;
  if (!encode_operand(&ta, g.A, g.M, g.K, TC_BM) || !encode_operand(&tw, g.B, N, g.K, N)) return false;
  gemm_tc_fwd_kernel<N><<<g.M / TC_BM, TC_THREADS, TcShape<N>::SMEM, s>>>(ta, tw, g.K, g.bias, g.zout, g.aout,
                                                                        g.ldc);
  tc_launch_count().fetch_add(1);
  return true;
}

// The layer on the tcgen05 path if selected and its shape allows; false: not launched.
inline bool forward_tc(const GemmArgs& g, cudaStream_t s) {
  if (forward_path().load() != TODGPU_MLP_TCGEN05 || g.K % TC_BK != 0 || g.M % TC_BM != 0 || g.lda != g.K ||
      g.ldb != g.K || g.ldc != g.N)
    return false;
  if (g.N == 256) return launch_tc<256>(g, s);
  if (g.N == 128) return launch_tc<128>(g, s);
  return false;
}

inline void forward_hidden(const Net& n, const Ws& w, long long M, bool keep_z, cudaStream_t s) {
  const Dims& d = n.d;
  features_kernel<<<grid1d(M * d.F, 256), 256, 0, s>>>(w.x, M, n.freq, d.F, w.feat);
  for (int l = 0; l < d.D; ++l) {
    GemmArgs g{};
    g.A = l == 0 ? w.feat : w.a + (long long)(l - 1) * M * d.H;
    g.lda = d.K(l);
    g.B = n.pb + n.off.w[l];
    g.ldb = d.K(l);
    g.M = (int)M;
    g.N = d.H;
    g.K = d.K(l);
    g.bias = n.p + n.off.b[l];
    g.zout = keep_z ? w.z + (long long)l * M * d.H : nullptr;
    g.aout = w.a + (long long)l * M * d.H;
    g.ldc = d.H;
    if (!forward_tc(g, s)) gemm<0, 0, EPI_FWD>(g, 1, s);
  }
}

template <int O>
void head(const Net& n, const Ws& w, long long M, const HeadOut& h, cudaStream_t s) {
  const Dims& d = n.d;
  const bf16* act = w.a + (long long)(d.D - 1) * M * d.H;
  head_kernel<O><<<grid1d(M * 32, 256), 256, 0, s>>>(act, M, d.H, n.pb + n.off.w[d.D], n.p + n.off.b[d.D], h);
}

inline void head_dispatch(const Net& n, const Ws& w, long long M, const HeadOut& h, cudaStream_t s) {
  switch (n.d.O) {
    case 1: head<1>(n, w, M, h, s); break;
    case 2: head<2>(n, w, M, h, s); break;
    case 3: head<3>(n, w, M, h, s); break;
    default: head<4>(n, w, M, h, s); break;
  }
}

template <int O>
void head_backward(const Net& n, const Ws& w, long long M, int splits, cudaStream_t s) {
  const Dims& d = n.d;
  const long long last = (long long)(d.D - 1) * M * d.H;
  const long long rows = M / splits;
  head_wgrad_kernel<O><<<splits, 256, 0, s>>>(w.y, w.a + last, rows, d.H, w.part);
  const long long cnt = (long long)O * d.H + O;  // head W then b, contiguous in the layout
  reduce_splits_kernel<<<grid1d(cnt, 256), 256, 0, s>>>(w.part, splits, cnt, n.grad + n.off.w[d.D]);
  head_bwd_kernel<O><<<grid1d(M * d.H, 256), 256, 0, s>>>(w.y, M, d.H, n.pb + n.off.w[d.D], w.z + last, w.dz);
}

// loss and full gradient of the batch in w.x (inputs) against target (M, O).
inline void loss_grad(const Net& n, const Ws& w, long long M, const float* target, float* loss_out, cudaStream_t s) {
  const Dims& d = n.d;
  forward_hidden(n, w, M, true, s);
  HeadOut h{};
  h.target = target;
  h.dy = w.y;
  h.loss = w.loss;
  h.grad_scale = 2.0f / (float)(M * d.O);
  head_dispatch(n, w, M, h, s);
  loss_mean_kernel<<<1, kThreads, 0, s>>>(w.loss, M, 1.0f / (float)(M * d.O), loss_out ? loss_out : w.loss + M);
  const int splits = splits_for(M);
  switch (d.O) {
    case 1: head_backward<1>(n, w, M, splits, s); break;
    case 2: head_backward<2>(n, w, M, splits, s); break;
    case 3: head_backward<3>(n, w, M, splits, s); break;
    default: head_backward<4>(n, w, M, splits, s); break;
  }
  // hidden layers, last to first; dz ping-pongs between two buffers
  for (int l = d.D - 1; l >= 0; --l) {
    bf16* dz = w.dz + (long long)((d.D - 1 - l) & 1) * M * d.H;
    bf16* dz_prev = w.dz + (long long)((d.D - l) & 1) * M * d.H;
    const bf16* a_in = l == 0 ? w.feat : w.a + (long long)(l - 1) * M * d.H;
    const int K = d.K(l);
    // dW_l(n, k) = sum_m dz(m, n) a_in(m, k): split over m
    GemmArgs g{};
    g.A = dz;
    g.lda = d.H;
    g.B = a_in;
    g.ldb = K;
    g.M = d.H;
    g.N = K;
    g.K = (int)(M / splits);
    g.cout = w.part;
    g.ldc = K;
    gemm<1, 1, EPI_PART>(g, splits, s);
    const long long cnt = (long long)d.H * K;
    reduce_splits_kernel<<<grid1d(cnt, 256), 256, 0, s>>>(w.part, splits, cnt, n.grad + n.off.w[l]);
    colsum_kernel<<<splits, 256, 0, s>>>(dz, M / splits, d.H, w.part);
    reduce_splits_kernel<<<grid1d(d.H, 256), 256, 0, s>>>(w.part, splits, d.H, n.grad + n.off.b[l]);
    if (l > 0) {
      // dz_prev(m, k) = (sum_n dz(m, n) W_l(n, k)) silu'(z_{l-1}(m, k))
      GemmArgs b{};
      b.A = dz;
      b.lda = d.H;
      b.B = n.pb + n.off.w[l];
      b.ldb = K;
      b.M = (int)M;
      b.N = K;
      b.K = d.H;
      b.zin = w.z + (long long)(l - 1) * M * d.H;
      b.aout = dz_prev;
      b.ldc = K;
      gemm<0, 1, EPI_BWD>(b, 1, s);
    }
  }
}

inline void adam(const Net& n, long long step, float lr, float b1, float b2, float eps, cudaStream_t s) {
  const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
  adam_kernel<<<grid1d(n.off.total, 256), 256, 0, s>>>(n.p, n.pb, n.am, n.av, n.grad, n.off.total, lr, b1, b2, eps,
                                                       bc1, bc2);
}

}  // namespace mlp
}  // namespace todgpu

using namespace todgpu;
using namespace todgpu::mlp;

namespace {

int check_dims(const todgpu_mlp* m, Dims& d) {
  if (!m) return fail(TODGPU_EINVAL, "NULL network descriptor");
  d = Dims{m->n_freq, m->width, m->depth, m->n_out};
  if (d.F <= 0 || (2 * d.F) % 128 != 0) return fail(TODGPU_ESHAPE, "n_freq must be a positive multiple of 64");
  if (d.H <= 0 || d.H % 128 != 0) return fail(TODGPU_ESHAPE, "width must be a positive multiple of 128");
  if (d.D < 1 || d.D > kMaxDepth) return fail(TODGPU_ESHAPE, "depth must be in [1, 8]");
  if (d.O < 1 || d.O > kMaxOut) return fail(TODGPU_ESHAPE, "n_out must be in [1, 4]");
  return TODGPU_OK;
}

int check_net(const todgpu_mlp* m, Dims& d, bool training) {
  const int rc = check_dims(m, d);
  if (rc) return rc;
  if (!m->freq || !m->params || !m->params_bf16) return fail(TODGPU_EINVAL, "NULL network buffer");
  if (training && (!m->grad || !m->adam_m || !m->adam_v)) return fail(TODGPU_EINVAL, "NULL training buffer");
  return TODGPU_OK;
}

Net make_net(const todgpu_mlp* m, const Dims& d) {
  return Net{d, param_offsets(d), m->freq, m->params, static_cast<bf16*>(m->params_bf16), m->grad, m->adam_m,
             m->adam_v};
}

int check_ws(const Dims& d, long long M, const void* ws, size_t bytes) {
  if (M <= 0 || M % BM != 0) return fail(TODGPU_ESHAPE, "batch rows must be a positive multiple of 128");
  if (M > (1LL << 30)) return fail(TODGPU_ESHAPE, "batch rows too large");
  if (!ws) return fail(TODGPU_EINVAL, "NULL workspace");
  long long o[R_COUNT + 1];
  ws_offsets(d, M, o);
  if ((long long)bytes < o[R_COUNT]) return fail(TODGPU_ESHAPE, "workspace too small");
  return TODGPU_OK;
}

int finish(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, what);
}

}  // namespace

extern "C" int64_t todgpu_mlp_param_count(const todgpu_mlp* m) {
  Dims d;
  if (check_dims(m, d)) return -1;
  return param_offsets(d).total;
}

extern "C" int todgpu_mlp_param_offsets(const todgpu_mlp* m, int64_t* w_off, int64_t* b_off) {
  Dims d;
  const int rc = check_dims(m, d);
  if (rc) return rc;
  if (!w_off || !b_off) return fail(TODGPU_EINVAL, "NULL output");
  const Offsets o = param_offsets(d);
  for (int l = 0; l <= d.D; ++l) {
    w_off[l] = o.w[l];
    b_off[l] = o.b[l];
  }
  return TODGPU_OK;
}

extern "C" size_t todgpu_mlp_workspace_bytes(const todgpu_mlp* m, int64_t rows) {
  Dims d;
  if (check_dims(m, d) || rows <= 0 || rows % BM != 0) return 0;
  long long o[R_COUNT + 1];
  ws_offsets(d, rows, o);
  return (size_t)o[R_COUNT];
}

extern "C" int todgpu_mlp_workspace_offsets(const todgpu_mlp* m, int64_t rows, int64_t* offsets) {
  Dims d;
  const int rc = check_dims(m, d);
  if (rc) return rc;
  if (rows <= 0 || rows % BM != 0) return fail(TODGPU_ESHAPE, "rows must be a positive multiple of 128");
  if (!offsets) return fail(TODGPU_EINVAL, "NULL output");
  long long o[R_COUNT + 1];
  ws_offsets(d, rows, o);
  for (int i = 0; i <= R_COUNT; ++i) offsets[i] = o[i];
  return TODGPU_OK;
}

extern "C" int todgpu_mlp_sync_bf16(const todgpu_mlp* m, void* stream) {
  Dims d;
  const int rc = check_net(m, d, false);
  if (rc) return rc;
  const long long n = param_offsets(d).total;
  to_bf16_kernel<<<grid1d(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      m->params, static_cast<bf16*>(m->params_bf16), n);
  return finish("mlp bf16 copy");
}

extern "C" int todgpu_mlp_inputs(const void* theta, const void* phi, const void* psi, int32_t angles_dtype, int64_t n,
                                 int64_t rows, float* x, void* stream) {
  if (n < 0 || rows < n) return fail(TODGPU_ESHAPE, "need 0 <= n <= rows");
  if (!x || (n > 0 && (!theta || !phi || !psi))) return fail(TODGPU_EINVAL, "NULL pointer");
  if (angles_dtype != TODGPU_F32 && angles_dtype != TODGPU_F64)
    return fail(TODGPU_EDTYPE, "angles_dtype must be TODGPU_F32 or TODGPU_F64");
  if (rows == 0) return TODGPU_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (angles_dtype == TODGPU_F32)
    inputs_kernel<float><<<grid1d(rows, 256), 256, 0, s>>>(static_cast<const float*>(theta),
                                                           static_cast<const float*>(phi),
                                                           static_cast<const float*>(psi), n, rows, x);
  else
    inputs_kernel<double><<<grid1d(rows, 256), 256, 0, s>>>(static_cast<const double*>(theta),
                                                            static_cast<const double*>(phi),
                                                            static_cast<const double*>(psi), n, rows, x);
  return finish("mlp inputs");
}

extern "C" int todgpu_mlp_forward(const todgpu_mlp* m, const float* x, int64_t rows, void* ws, size_t ws_bytes,
                                  float* y, void* stream) {
  Dims d;
  int rc = check_net(m, d, false);
  if (rc) return rc;
  if ((rc = check_ws(d, rows, ws, ws_bytes))) return rc;
  if (!x || !y) return fail(TODGPU_EINVAL, "NULL pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Net n = make_net(m, d);
  const Ws w = ws_view(d, rows, ws);
  cudaMemcpyAsync(w.x, x, sizeof(float) * kIn * rows, cudaMemcpyDeviceToDevice, s);
  forward_hidden(n, w, rows, false, s);
  HeadOut h{};
  h.y = y;
  head_dispatch(n, w, rows, h, s);
  return finish("mlp forward");
}

extern "C" int todgpu_mlp_loss_grad(const todgpu_mlp* m, const float* x, const float* target, int64_t rows, void* ws,
                                    size_t ws_bytes, float* loss, void* stream) {
  Dims d;
  int rc = check_net(m, d, true);
  if (rc) return rc;
  if ((rc = check_ws(d, rows, ws, ws_bytes))) return rc;
  if (!x || !target) return fail(TODGPU_EINVAL, "NULL pointer");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Net n = make_net(m, d);
  const Ws w = ws_view(d, rows, ws);
  cudaMemcpyAsync(w.x, x, sizeof(float) * kIn * rows, cudaMemcpyDeviceToDevice, s);
  loss_grad(n, w, rows, target, loss, s);
  return finish("mlp loss/grad");
}

extern "C" int todgpu_mlp_adam(const todgpu_mlp* m, int64_t step, float lr, float beta1, float beta2, float eps,
                               void* stream) {
  Dims d;
  const int rc = check_net(m, d, true);
  if (rc) return rc;
  if (step < 1) return fail(TODGPU_EINVAL, "step counts from 1");
  adam(make_net(m, d), step, lr, beta1, beta2, eps, static_cast<cudaStream_t>(stream));
  return finish("mlp adam");
}

extern "C" int todgpu_mlp_train(const todgpu_mlp* m, const float* x, const float* target, int64_t n_rows,
                                int64_t batch, int64_t first_step, int64_t n_steps, int64_t total_steps, float lr_max,
                                float lr_min, void* ws, size_t ws_bytes, float* loss_per_step, void* stream) {
  Dims d;
  int rc = check_net(m, d, true);
  if (rc) return rc;
  if ((rc = check_ws(d, batch, ws, ws_bytes))) return rc;
  if (!x || !target) return fail(TODGPU_EINVAL, "NULL pointer");
  if (n_rows < batch || n_rows % batch != 0) return fail(TODGPU_ESHAPE, "n_rows must be a multiple of batch");
  if (first_step < 0 || n_steps < 0 || total_steps < first_step + n_steps)
    return fail(TODGPU_EINVAL, "bad step range");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Net n = make_net(m, d);
  const Ws w = ws_view(d, batch, ws);
  const long long nb = n_rows / batch;
  for (long long i = 0; i < n_steps; ++i) {
    const long long step = first_step + i;  // 0-based
    const long long r0 = (step % nb) * batch;
    cudaMemcpyAsync(w.x, x + r0 * kIn, sizeof(float) * kIn * batch, cudaMemcpyDeviceToDevice, s);
    loss_grad(n, w, batch, target + r0 * d.O, loss_per_step ? loss_per_step + i : nullptr, s);
    const double c = 0.5 * (1.0 + std::cos(kPi * (double)step / (double)std::max<int64_t>(1, total_steps)));
    const float lr = (float)(lr_min + (lr_max - lr_min) * c);
    adam(n, step + 1, lr, 0.9f, 0.999f, 1e-8f, s);
  }
  return finish("mlp train");
}

extern "C" int todgpu_tail_accumulate(const todgpu_mlp* m, const void* theta, const void* phi, const void* psi,
                                      int32_t angles_dtype, int64_t B, const int32_t* rows, const double* scale,
                                      const double* shift, double* tod, int64_t tod_stride, int64_t chunk, void* ws,
                                      size_t ws_bytes, void* stream) {
  Dims d;
  int rc = check_net(m, d, false);
  if (rc) return rc;
  if ((rc = check_ws(d, chunk, ws, ws_bytes))) return rc;
  if (B < 0) return fail(TODGPU_ESHAPE, "B must be >= 0");
  if (!rows || !scale || !shift || (B > 0 && (!tod || !theta || !phi || !psi)))
    return fail(TODGPU_EINVAL, "NULL pointer");
  if (angles_dtype != TODGPU_F32 && angles_dtype != TODGPU_F64) return fail(TODGPU_EDTYPE, "bad angles_dtype");
  if (tod_stride < B) return fail(TODGPU_ESHAPE, "tod_stride < B");
  for (int o = 0; o < d.O; ++o)
    if (rows[o] < 0) return fail(TODGPU_ESHAPE, "negative output row");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Net n = make_net(m, d);
  const Ws w = ws_view(d, chunk, ws);
  const size_t esz = angles_dtype == TODGPU_F32 ? 4 : 8;
  HeadOut h{};
  h.tod = tod;
  h.tod_stride = tod_stride;
  for (int o = 0; o < d.O; ++o) {
    h.rows[o] = rows[o];
    h.scale[o] = scale[o];
    h.shift[o] = shift[o];
  }
  for (long long b0 = 0; b0 < B; b0 += chunk) {
    const long long nv = std::min<long long>(chunk, B - b0);
    const char* th = static_cast<const char*>(theta) + b0 * esz;
    const char* ph = static_cast<const char*>(phi) + b0 * esz;
    const char* ps = static_cast<const char*>(psi) + b0 * esz;
    if (angles_dtype == TODGPU_F32)
      inputs_kernel<float><<<grid1d(chunk, 256), 256, 0, s>>>(reinterpret_cast<const float*>(th),
                                                              reinterpret_cast<const float*>(ph),
                                                              reinterpret_cast<const float*>(ps), nv, chunk, w.x);
    else
      inputs_kernel<double><<<grid1d(chunk, 256), 256, 0, s>>>(reinterpret_cast<const double*>(th),
                                                               reinterpret_cast<const double*>(ph),
                                                               reinterpret_cast<const double*>(ps), nv, chunk, w.x);
    forward_hidden(n, w, chunk, false, s);
    h.b0 = b0;
    h.n_valid = nv;
    head_dispatch(n, w, chunk, h, s);
  }
  return finish("tail accumulate");
}

extern "C" int todgpu_mlp_set_forward_path(int32_t path) {
  if (path != TODGPU_MLP_TCGEN05 && path != TODGPU_MLP_MMA_SYNC) return fail(TODGPU_EINVAL, "unknown forward path");
  return forward_path().exchange(path);
}

extern "C" int64_t todgpu_mlp_wait_timeouts(void) {
  unsigned int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_tc_timeouts, sizeof(v)) != cudaSuccess) return -1;
  return (int64_t)v;
}

extern "C" int64_t todgpu_mlp_tcgen05_launches(void) { return tc_launch_count().load(); }
