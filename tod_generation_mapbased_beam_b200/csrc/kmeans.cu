// kmeans.cu -- weighted spherical k-means of beam pixels on the GPU, the
// clustering behind beam_cluster.cluster_beam_pixels (beam_cluster.py:70-188):
// k-means++ seeding and the assignment / weighted-centroid iterations.
//
// * Similarities are v . c with the products accumulated as
//   fma(v2, c2, fma(v1, c1, v0 c0)), the order a BLAS matrix product with
//   fused multiply-adds uses; argmax keeps the first maximum, like numpy.
// * The per-cluster sums (weights, weighted vectors) are taken in pixel order
//   for every cluster, as numpy's bincount does: a stable counting sort of
//   the pixels by label (per-chunk histograms, a per-cluster scan over the
//   chunks, a warp-sequential stable scatter) and then one sequential sum per
//   cluster -- deterministic and equal to the sequential sums bit for bit.
// * k-means++ seeding draws index i with probability p_i / sum p (p_i =
//   w_i max(1 - nearest_cos_i, 0)^2) as the first i with
//   cumsum(p)_i / sum(p) > u for a uniform u supplied by the caller (so the
//   caller's random stream decides); the cumulative sums are taken per block
//   and then across blocks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "gather_impl.cuh"

namespace todgpu {
namespace km {

constexpr int kThreads = 256;
constexpr int kChunk = 2048;         // pixels per histogram/scatter chunk
constexpr int kMaxClusters = 8192;   // shared-memory counters of one chunk
constexpr int kCentTile = 2048;      // centroids staged in shared memory at a time

__device__ __forceinline__ double dot3(const double* v, double c0, double c1, double c2) {
  return fma(v[2], c2, fma(v[1], c1, v[0] * c0));
}

// labels[i] = argmax_k v_i . c_k (first maximum), best[i] = that maximum
__global__ void assign_kernel(const double* vec, long long S, const double* cent, int K, int* labels, double* best) {
  __shared__ double sc[kCentTile * 3];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double v[3] = {0.0, 0.0, 0.0};
  if (i < S) {
    v[0] = vec[3 * i];
    v[1] = vec[3 * i + 1];
    v[2] = vec[3 * i + 2];
  }
  double bs = -INFINITY;
  int bl = 0;
  for (int k0 = 0; k0 < K; k0 += kCentTile) {
    const int nk = min(kCentTile, K - k0);
    __syncthreads();
    for (int t = threadIdx.x; t < 3 * nk; t += blockDim.x) sc[t] = cent[3LL * k0 + t];
    __syncthreads();
    for (int k = 0; k < nk; ++k) {
      const double s = dot3(v, sc[3 * k], sc[3 * k + 1], sc[3 * k + 2]);
      if (s > bs) {
        bs = s;
        bl = k0 + k;
      }
    }
  }
  if (i < S) {
    labels[i] = bl;
    best[i] = bs;
  }
}

// counts[c * K + k] = pixels of chunk c with label k
__global__ void chunk_hist_kernel(const int* labels, long long S, int K, int* counts) {
  __shared__ int h[kMaxClusters];
  for (int k = threadIdx.x; k < K; k += blockDim.x) h[k] = 0;
  __syncthreads();
  const long long c0 = (long long)blockIdx.x * kChunk;
  for (long long i = c0 + threadIdx.x; i < min(S, c0 + kChunk); i += blockDim.x) atomicAdd(&h[labels[i]], 1);
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) counts[(long long)blockIdx.x * K + k] = h[k];
}

// per cluster: base[c * K + k] = pixels of label k in chunks before c; total[k]
__global__ void chunk_scan_kernel(int* counts, int nchunks, int K, int* total) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  int run = 0;
  for (int c = 0; c < nchunks; ++c) {
    const int n = counts[(long long)c * K + k];
    counts[(long long)c * K + k] = run;
    run += n;
  }
  total[k] = run;
}

// offsets[k] = sum of total[0..k) (one block, K <= kMaxClusters)
__global__ void offsets_kernel(const int* total, int K, int* offsets) {
  __shared__ int part[kThreads];
  const int per = (K + blockDim.x - 1) / blockDim.x;
  const int k0 = threadIdx.x * per, k1 = min(K, k0 + per);
  int s = 0;
  for (int k = k0; k < k1; ++k) s += total[k];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const int n = part[t];
      part[t] = run;
      run += n;
    }
    offsets[K] = run;
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int k = k0; k < k1; ++k) {
    offsets[k] = run;
    run += total[k];
  }
}

// Stable scatter of chunk c: one warp walks the chunk in index order, 32 pixels
// at a time; pixels of one label in a step take consecutive slots in lane order.
__global__ void scatter_kernel(const int* labels, long long S, int K, const int* base, const int* offsets,
                               int* order) {
  __shared__ int next[kMaxClusters];
  for (int k = threadIdx.x; k < K; k += blockDim.x) next[k] = offsets[k] + base[(long long)blockIdx.x * K + k];
  __syncthreads();
  if (threadIdx.x >= 32) return;
  const int lane = threadIdx.x;
  const long long c0 = (long long)blockIdx.x * kChunk, c1 = min(S, c0 + kChunk);
  for (long long i0 = c0; i0 < c1; i0 += 32) {
    const long long i = i0 + lane;
    const bool valid = i < c1;
    const int lab = valid ? labels[i] : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, lab);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int slot = valid ? next[lab] + rank : 0;
    __syncwarp();
    if (valid) order[slot] = (int)i;
    const int leader = __ffs(peers) - 1;
    if (valid && lane == leader) next[lab] += __popc(peers);
    __syncwarp();
  }
}

// sums[4 k ..] = (sum w x, sum w y, sum w z, sum w) over cluster k's pixels in
// increasing pixel order (products w * v rounded first, then added in order)
__global__ void cluster_sums_kernel(const double* vec, const double* w, const int* order, const int* offsets, int K,
                                    double* sums) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double sx = 0.0, sy = 0.0, sz = 0.0, sw = 0.0;
  for (int j = offsets[k]; j < offsets[k + 1]; ++j) {
    const long long i = order[j];
    const double wi = w[i];
    sw += wi;
    sx += wi * vec[3 * i];
    sy += wi * vec[3 * i + 1];
    sz += wi * vec[3 * i + 2];
  }
  sums[4 * k] = sx;
  sums[4 * k + 1] = sy;
  sums[4 * k + 2] = sz;
  sums[4 * k + 3] = sw;
}

// First index of the minimum of best[0..S) (one block).
__global__ void argmin_kernel(const double* best, long long S, long long* out) {
  __shared__ double sv[kThreads];
  __shared__ long long si[kThreads];
  double bv = INFINITY;
  long long bi = S;
  for (long long i = threadIdx.x; i < S; i += blockDim.x) {
    const double v = best[i];
    if (v < bv) {
      bv = v;
      bi = i;
    }
  }
  sv[threadIdx.x] = bv;
  si[threadIdx.x] = bi;
  __syncthreads();
  for (int d = blockDim.x / 2; d > 0; d >>= 1) {
    if ((int)threadIdx.x < d) {
      const double v = sv[threadIdx.x + d];
      const long long j = si[threadIdx.x + d];
      if (v < sv[threadIdx.x] || (v == sv[threadIdx.x] && j < si[threadIdx.x])) {
        sv[threadIdx.x] = v;
        si[threadIdx.x] = j;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = si[0] < S ? si[0] : 0;
}

// ---- k-means++ seeding ------------------------------------------------------
// Step k: nearest[i] = max(nearest[i], v_i . c_{k-1}) (k >= 1), p_i as above
// (p_i = w_i at k = 0), block sums of p.
__global__ void seed_weights_kernel(const double* vec, const double* w, long long S, double* nearest,
                                    const double* cent, int k, double* p, double* block_sums) {
  __shared__ double red[kThreads];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double pi = 0.0;
  if (i < S) {
    if (k == 0) {
      pi = w[i];
    } else {
      const double* c = cent + 3LL * (k - 1);
      const double s = dot3(vec + 3 * i, c[0], c[1], c[2]);
      double nc = (k == 1) ? s : nearest[i];
      if (k > 1 && s > nc) nc = s;
      nearest[i] = nc;
      const double d = max(1.0 - nc, 0.0);
      pi = w[i] * (d * d);
    }
    p[i] = pi;
  }
  // block sum in a fixed order
  red[threadIdx.x] = pi;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) s += red[t];
    block_sums[blockIdx.x] = s;
  }
}

// One block: the drawn index for uniform u -- the first i with
// cumsum(p)_i / total > u -- then c_k = v_i.  When every p_i is 0 the weights
// w are used instead (the caller's fallback to the initial probabilities).
__global__ void seed_pick_kernel(const double* vec, const double* w, long long S, const double* p,
                                 const double* block_sums, int nblocks, double u, int k, double* cent,
                                 long long* chosen) {
  __shared__ double s_prefix;
  __shared__ int s_block;
  __shared__ int s_zero;
  if (threadIdx.x == 0) {
    double total = 0.0;
    for (int b = 0; b < nblocks; ++b) total += block_sums[b];
    s_zero = !(total > 0.0);
    s_block = -1;
    s_prefix = 0.0;
    if (!s_zero) {
      double run = 0.0;
      for (int b = 0; b < nblocks; ++b) {
        const double nxt = run + block_sums[b];
        if (nxt / total > u) {
          s_block = b;
          s_prefix = run;
          break;
        }
        run = nxt;
      }
      if (s_block < 0) {  // u at or above the rounded total: the last positive block
        run = 0.0;
        for (int b = 0; b < nblocks; ++b) {
          if (block_sums[b] > 0.0) {
            s_block = b;
            s_prefix = run;
          }
          run += block_sums[b];
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  long long pick = S - 1;
  if (s_zero) {
    // fall back to the weights themselves (sequential, one thread)
    double total = 0.0;
    for (long long i = 0; i < S; ++i) total += w[i];
    double run = 0.0;
    for (long long i = 0; i < S; ++i) {
      run += w[i];
      if (run / total > u) {
        pick = i;
        break;
      }
    }
  } else {
    double total = 0.0;
    for (int b = 0; b < nblocks; ++b) total += block_sums[b];
    double run = s_prefix;
    const long long i0 = (long long)s_block * kThreads, i1 = min(S, i0 + kThreads);
    pick = i1 - 1;
    for (long long i = i0; i < i1; ++i) {
      run += p[i];
      if (run / total > u) {
        pick = i;
        break;
      }
    }
  }
  chosen[k] = pick;
  cent[3LL * k] = vec[3 * pick];
  cent[3LL * k + 1] = vec[3 * pick + 1];
  cent[3LL * k + 2] = vec[3 * pick + 2];
}

inline unsigned blocks_for(long long n, int t) { return (unsigned)std::max(1LL, (n + t - 1) / t); }

}  // namespace km
}  // namespace todgpu

using namespace todgpu;
using namespace todgpu::km;

namespace {

int check_sk(long long S, int K) {
  if (S < 1 || S > (1LL << 31) - 1) return fail(TODGPU_ESHAPE, "pixel count must be in [1, 2^31)");
  if (K < 1 || K > kMaxClusters) return fail(TODGPU_ESHAPE, "cluster count must be in [1, 8192]");
  return TODGPU_OK;
}

int done(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TODGPU_OK : cuda_fail(e, what);
}

}  // namespace

extern "C" size_t todgpu_kmeans_workspace_bytes(int64_t S, int32_t K) {
  if (S < 1 || K < 1 || K > kMaxClusters) return 0;
  const long long nchunks = (S + kChunk - 1) / kChunk;
  const long long nblk = (S + kThreads - 1) / kThreads;
  const long long ints = nchunks * K + K + (K + 1) + S;  // base/counts, total, offsets, order
  const long long dbl = S + S + nblk;                     // nearest, p, block sums
  return (size_t)(ints * 4 + 64 + dbl * 8 + 64);
}

extern "C" int todgpu_kmeans_seed(const double* vec, const double* w, int64_t S, int32_t K, const double* uniforms,
                                  double* centroids, int64_t* chosen, void* ws, size_t ws_bytes, void* stream) {
  int rc = check_sk(S, K);
  if (rc) return rc;
  if (!vec || !w || !uniforms || !centroids || !chosen || !ws) return fail(TODGPU_EINVAL, "NULL pointer");
  if (ws_bytes < todgpu_kmeans_workspace_bytes(S, K)) return fail(TODGPU_ESHAPE, "workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long nchunks = (S + kChunk - 1) / kChunk;
  const long long nblk = (S + kThreads - 1) / kThreads;
  char* b = static_cast<char*>(ws);
  double* dws = reinterpret_cast<double*>(b + ((nchunks * K + K + (K + 1) + S) * 4 + 64) / 8 * 8);
  double* nearest = dws;
  double* p = dws + S;
  double* bsum = dws + 2 * S;
  for (int k = 0; k < K; ++k) {
    seed_weights_kernel<<<(unsigned)nblk, kThreads, 0, s>>>(vec, w, S, nearest, centroids, k, p, bsum);
    seed_pick_kernel<<<1, 32, 0, s>>>(vec, w, S, p, bsum, (int)nblk, uniforms[k], k, centroids,
                                      reinterpret_cast<long long*>(chosen));
  }
  return done("kmeans seeding");
}

extern "C" int todgpu_kmeans_assign(const double* vec, int64_t S, const double* centroids, int32_t K, int32_t* labels,
                                    double* best, void* stream) {
  int rc = check_sk(S, K);
  if (rc) return rc;
  if (!vec || !centroids || !labels || !best) return fail(TODGPU_EINVAL, "NULL pointer");
  assign_kernel<<<blocks_for(S, kThreads), kThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      vec, S, centroids, K, reinterpret_cast<int*>(labels), best);
  return done("kmeans assign");
}

extern "C" int todgpu_kmeans_sums(const double* vec, const double* w, const int32_t* labels, int64_t S, int32_t K,
                                  double* sums, void* ws, size_t ws_bytes, void* stream) {
  int rc = check_sk(S, K);
  if (rc) return rc;
  if (!vec || !w || !labels || !sums || !ws) return fail(TODGPU_EINVAL, "NULL pointer");
  if (ws_bytes < todgpu_kmeans_workspace_bytes(S, K)) return fail(TODGPU_ESHAPE, "workspace too small");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long nchunks = (S + kChunk - 1) / kChunk;
  int* counts = static_cast<int*>(ws);
  int* total = counts + nchunks * K;
  int* offsets = total + K;
  int* order = offsets + (K + 1);
  const int* lab = reinterpret_cast<const int*>(labels);
  chunk_hist_kernel<<<(unsigned)nchunks, kThreads, 0, s>>>(lab, S, K, counts);
  chunk_scan_kernel<<<blocks_for(K, kThreads), kThreads, 0, s>>>(counts, (int)nchunks, K, total);
  offsets_kernel<<<1, kThreads, 0, s>>>(total, K, offsets);
  scatter_kernel<<<(unsigned)nchunks, kThreads, 0, s>>>(lab, S, K, counts, offsets, order);
  cluster_sums_kernel<<<blocks_for(K, 128), 128, 0, s>>>(vec, w, order, offsets, K, sums);
  return done("kmeans sums");
}

extern "C" int todgpu_kmeans_argmin(const double* best, int64_t S, int64_t* index, void* stream) {
  if (S < 1) return fail(TODGPU_ESHAPE, "S must be >= 1");
  if (!best || !index) return fail(TODGPU_EINVAL, "NULL pointer");
  argmin_kernel<<<1, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(best, S,
                                                                        reinterpret_cast<long long*>(index));
  return done("kmeans argmin");
}
