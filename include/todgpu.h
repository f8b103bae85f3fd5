/*
 * todgpu.h -- C ABI of the B200 beam-convolution TOD library (libtodgpu.so).
 *
 * Plain pointers and sizes only.  Device pointers are CUDA device addresses
 * on the current device; `stream` is a cudaStream_t passed as void* (NULL =
 * legacy default stream).  Every entry point returns 0 (TODGPU_OK) or a
 * negative TODGPU_E* code; todgpu_last_error_string() describes the last
 * failure of the calling thread.
 *
 * Each declaration names the reference interface it replaces
 * (ArtemBasyrov/tod_generation_mapbased_beam, file:line).
 */
#ifndef TODGPU_H
#define TODGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TODGPU_ABI_VERSION 1

/* Status codes. */
#define TODGPU_OK 0
#define TODGPU_EINVAL -1      /* bad argument (NULL pointer, unknown enum)      */
#define TODGPU_ENSIDE -2      /* nside outside [1, 8192]                         */
#define TODGPU_ESHAPE -3      /* B, S or C out of range, c_q/c_u inconsistent    */
#define TODGPU_EDTYPE -4      /* unsupported dtype combination                   */
#define TODGPU_ECUDA -5       /* a CUDA runtime call failed                      */
#define TODGPU_EABI -6        /* abi_version mismatch                            */

/* Interpolation modes (tod_core.py:114-119). */
#define TODGPU_BILINEAR 0
#define TODGPU_NEAREST 1

/* Flags (todgpu_gather_args.flags). */
#define TODGPU_FLAG_NO_TABLES 1 /* ignore ring_table: evaluate every stencil ring and spin-2
                                   angle directly (same results, slower) */
#define TODGPU_FLAG_NO_BEAM_STAGE 2 /* read the beam from global memory even when the launch
                                       could hold it in shared memory (same results) */
#define TODGPU_FLAG_WIDE_CTAS 4 /* launch 256-thread CTAs even where the spin-2 table asked
                                   for (tab_slots) fits 128-thread CTAs at 8 per SM
                                   (same results) */

/* Element types. */
#define TODGPU_F32 0
#define TODGPU_F64 1
/* params_dtype: pointing given as angles, rotation derived on the device. */
#define TODGPU_ANGLES 2
/* map_dtype of the precision form: one record of 4 components per pixel,
 * float32 (16 B) or bfloat16 (8 B), made by todgpu_pack_map.  With a packed
 * map the spin-2 angles are kept in float32 and the sum over beam pixels is
 * float32 with Kahan compensation; rotation, pixel choice and weights stay
 * float64. */
#define TODGPU_PACKED_F32 2
#define TODGPU_PACKED_BF16 3
/* map_dtype: one record of 4 float64 components per pixel (32 B, 16-byte
 * aligned), made by todgpu_pack_map: the float64 path with a pixel's I/Q/U
 * side by side -- same values and arithmetic as a planar float64 map, so the
 * same results bit for bit, with one memory sector per stencil pixel. */
#define TODGPU_PACKED_F64 4

/*
 * Arguments of one fused gather/accumulate call: one beam entry over a batch
 * of B samples, accumulating into tod (tod[c*tod_stride + b] += ...).
 *
 * params_dtype = TODGPU_F32: vec_orig and the six per-sample parameter arrays
 *   are float32 and are combined with the reference's operand types (a float32
 *   recentre step, float64 elsewhere); this is the bit-parity form.
 *   bore_phi (optional, (B,) float32) holds atan2f(ax_pts[b,1], ax_pts[b,0])
 *   from the host C library (todgpu_boresight_phi_host): the reference
 *   computes that longitude with the host libm's float32 atan2, which the
 *   device's atan2 does not reproduce bit for bit.  When bore_phi is NULL the
 *   device rounds its float64 atan2 to float32 instead (Q/U may then differ
 *   from the reference by ~1e-7 relative on some samples).
 * params_dtype = TODGPU_F64: all float64, bore_phi ignored (precision form).
 * params_dtype = TODGPU_ANGLES: the seven parameter arrays are not read;
 *   theta, phi, psi (B,) (angles_dtype float32 or float64) and the beam centre
 *   (center_phi, center_theta) give the pointing, and every CTA derives the
 *   sample's rotation in float64 on the device (the steps of
 *   precompute_rotation_vector_batch, tod_rotations.py:219-303, and
 *   _rotation_params, :306-333, with psi_b - beta as the roll, gridint.py:281,
 *   and no float32 rounding); vec_orig is then float64 (S, 3).
 *
 * map: planar (C, map_stride) of map_dtype, RING order, map_stride >= 12*nside^2;
 *   or, for TODGPU_PACKED_*, N records of 4 components (map_stride ignored).
 * beam_vals: (S,) float32.  err_count: optional device uint64 counter that
 * receives the number of (b, s) terms skipped because a stencil pixel fell
 * outside the map (non-finite pointing); pass NULL to ignore.
 */
typedef struct todgpu_gather_args {
  int32_t abi_version;   /* TODGPU_ABI_VERSION */
  int32_t interp;        /* TODGPU_BILINEAR or TODGPU_NEAREST */
  int64_t nside;
  int64_t B;             /* samples */
  int64_t S;             /* beam pixels */
  int64_t C;             /* map components in this entry, 1..4 */
  int32_t c_q, c_u;      /* Q and U component positions in [0, C), or -1 */
  int32_t params_dtype;  /* TODGPU_F32 or TODGPU_F64 */
  int32_t map_dtype;     /* TODGPU_F32 or TODGPU_F64 */
  const void *vec_orig;  /* (S, 3) */
  const void *axes;      /* (B, 3) */
  const void *cos_a;     /* (B,) */
  const void *sin_a;     /* (B,) */
  const void *ax_pts;    /* (B, 3) */
  const void *cos_p;     /* (B,) */
  const void *sin_p;     /* (B,) */
  const float *bore_phi; /* (B,) or NULL */
  const float *beam_vals;/* (S,) */
  const void *map;       /* (C, map_stride) */
  int64_t map_stride;
  double *tod;           /* (C, tod_stride), accumulated in place */
  int64_t tod_stride;
  unsigned long long *err_count; /* optional */
  int32_t flags;         /* TODGPU_FLAG_* */
  int32_t tab_slots;     /* spin-2 table slots per sample in shared memory (with a
                            ring table and Q, U): 0 keeps the default of 2048 float64
                            / 4096 float32 pairs and 192 window rings; a footprint's
                            worth (about 1.05 (3.06 reach^2 nside^2 + 9 reach nside
                            + 12) + 32) also sizes the window-ring header (for a disc
                            of tab_slots / 3.2 pixels; 128-thread CTAs reserve 80
                            rings) and leaves the rest of the SM's memory to L1; up
                            to about 1500 float64 / 1900 float32 pairs the call runs
                            128-thread CTAs, 8 per SM.
                            Capped to what the kernel's CTAs per SM can share.  A
                            sample whose footprint needs more evaluates its spin-2
                            angles directly (same results).  Must be >= 0. */
  const void *ring_table;/* optional: table built by todgpu_ring_table_build for this
                            nside; NULL evaluates ring data and spin-2 angles directly */
  const void *theta;     /* (B,) boresight colatitude (TODGPU_ANGLES) */
  const void *phi;       /* (B,) boresight longitude */
  const void *psi;       /* (B,) polarisation angle psi_b */
  int32_t angles_dtype;  /* TODGPU_F32 or TODGPU_F64 */
  int32_t reserved2;
  double center_phi;     /* beam centre longitude = ra[centre] */
  double center_theta;   /* beam centre colatitude = pi/2 - dec[centre] */
} todgpu_gather_args;

/* Fused rotate -> HEALPix stencil -> spin-2 -> gather -> accumulate.
 * Replaces tod_bilinear._gather_accum_fused_jit (tod_bilinear.py:205-477)
 * and tod_nearest._gather_accum_nearest_jit (tod_nearest.py:21-158).
 * vec_orig must be aligned to its element size and beam_vals to 4 bytes;
 * S is at most 2^29.  When the beam fits in shared memory beside the spin-2
 * table, every CTA copies it there once per launch with bulk copies. */
int todgpu_gather_accum(const todgpu_gather_args *args, void *stream);

/* Number of bounded waits of the gather kernels (the beam's bulk copies into
 * shared memory) that ran out since the library was loaded: 0 in a healthy
 * run.  A CTA whose wait ran out copies the beam with plain loads instead,
 * so its results stay correct; the call's err_count, when given, counts it
 * too.  Reading it synchronises the device; -1 on a CUDA error.  No
 * counterpart in the reference. */
int64_t todgpu_gather_wait_timeouts(void);

/* Many jobs in one persistent launch: jobs[0 .. njobs) (a host array) are
 * independent gathers -- typically one detector each, with its own beam
 * (vec_orig, beam_vals, S), pointing (B samples) and output tod -- that share
 * interp, nside, the component layout (C, c_q, c_u), params_dtype, map_dtype
 * and flags.  Each job's samples are cut into tiles of `tile` samples (1 to
 * 2^24); the tiles of all jobs, numbered job by job, are dealt to the CTAs of
 * the persistent grid in turn (CTA k takes tiles k, k + G, ...), so that CTAs
 * running together work on neighbouring samples of one job.
 * Results equal one todgpu_gather_accum call per job.  Up to 96 jobs travel
 * in one launch's parameters; more are split over consecutive launches.
 * Replaces a loop of beam_tod_batch calls over detectors (the reference has
 * no batched-detector mode; gridint.py:284-296 loops over beam entries). */
int todgpu_gather_accum_batched(const todgpu_gather_args *jobs, int32_t njobs, int64_t tile,
                                void *stream);

/* The same fused gather/accumulate as todgpu_gather_accum, for callers that
 * cannot allocate device memory themselves -- for example a host application
 * whose device memory is owned by another framework's allocator, or a foreign-
 * language binding that can hand over existing buffers but has no way to
 * create new ones.  Instead of a caller-provided ring table it uses one built
 * into the library: a statically sized array (1.25 MiB, nside <= 4096) that every
 * GPU loading the library holds until the process exits.  args->ring_table is
 * ignored; nside > 4096 is rejected with TODGPU_ENSIDE.  Each call rebuilds
 * the table on `stream` for its own nside and beam before the gather, so no
 * state carries over between calls, but all calls share the one array: calls
 * that can overlap on the GPU (different streams or host threads) race and
 * must be serialised by the caller.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call before
 * any stream capture.  It allocates nothing.  No counterpart in the
 * reference. */
int todgpu_gather_accum_static(const todgpu_gather_args *args, void *stream);

/* Pointing preparation on the device (tod_rotations.py:219-333 with the roll
 * psi_b - beta of gridint.py:281, all in float64): for B samples (theta, phi,
 * psi) (angles_dtype TODGPU_F32 or TODGPU_F64) and the beam centre
 * (center_phi, center_theta), the rotation parameters axes (B, 3), cos_a,
 * sin_a, ax_pts (B, 3), cos_p, sin_p -- float64 device arrays -- exactly as
 * the TODGPU_ANGLES mode derives them inside the gather; a gather with
 * params_dtype = TODGPU_F64 on them gives the same TOD bit for bit.
 * Replaces the host step precompute_rotation_vector_batch + _rotation_params
 * for callers that keep the rotation on the GPU. */
int todgpu_pointing_params(const void *theta, const void *phi, const void *psi, int32_t angles_dtype, int64_t B,
                           double center_phi, double center_theta, double *axes, double *cos_a, double *sin_a,
                           double *ax_pts, double *cos_p, double *sin_p, void *stream);

/* Per-(b, s) bilinear stencil of the fused path: pix (4, B*S) int64 and
 * wgt (4, B*S) float64 with n = b*S + s.  Replaces the split reference path
 * tod_rotations._rodrigues_jit (tod_rotations.py:33-80) + vec2ang +
 * get_interp_weights_numba (numba_healpy.py:239-253) used by
 * tod_bilinear._gather_accum_jit (tod_bilinear.py:41-78).  Only the fields
 * nside, B, S, params_dtype and the seven parameter pointers of args are read. */
int todgpu_bilinear_stencils(const todgpu_gather_args *args, int64_t *pix, double *wgt,
                             void *stream);

/* hp.get_interp_weights in RING order on device arrays theta, phi (N,) f64
 * -> pix (4, N) int64, wgt (4, N) f64.
 * Replaces numba_healpy.get_interp_weights_numba (numba_healpy.py:239-253). */
int todgpu_get_interp_weights(int64_t nside, const double *theta, const double *phi, int64_t N,
                              int64_t *pix, double *wgt, void *stream);

/* Nearest RING pixel by the 4-candidate rule.
 * Replaces numba_healpy._ang2pix_ring_jit (numba_healpy.py:642-693). */
int todgpu_ang2pix(int64_t nside, const double *theta, const double *phi, int64_t N, int64_t *pix,
                   void *stream);

/* RING pixel centres. Replaces numba_healpy.pix2ang_numba (numba_healpy.py:622-635). */
int todgpu_pix2ang(int64_t nside, const int64_t *pix, int64_t N, double *theta, double *phi,
                   void *stream);

/* cos 2d / sin 2d of the spin-2 frame rotation on device arrays (N,).
 * Replaces tod_bilinear._spin2_cos2d_sin2d_jit (tod_bilinear.py:84-145). */
int todgpu_spin2(const double *z_pix, const double *sth_pix, const double *phi_pix,
                 const double *z_pts, const double *sth_pts, const double *phi_pts, int64_t N,
                 double *c2d, double *s2d, void *stream);

/* HOST function: out[b] = atan2f(ax_pts[3b+1], ax_pts[3b]) with the host C
 * library, multithreaded.  ax_pts and out are host pointers.  Produces the
 * boresight longitude the reference kernels compute in float32
 * (tod_bilinear.py:308, tod_nearest.py:87). */
int todgpu_boresight_phi_host(const float *ax_pts, int64_t B, float *out, int32_t nthreads);

/* Ring table: per-ring data of the RING scheme for one nside (ring z, acos z,
 * layout) and, for footprints of angular radius up to `reach` (radians), the
 * spin-2 table slots each ring needs.  todgpu_gather_accum reads it through
 * args->ring_table (lookups only; it is never written by the gather).  The
 * caller allocates `todgpu_ring_table_bytes(nside)` bytes of device memory
 * (16-byte aligned) and builds it once per (nside, reach) on `stream`.  A
 * beam wider than `reach` (its radius plus 4/nside) still runs, with the
 * spin-2 angles evaluated directly.  No counterpart in the reference, whose
 * kernels recompute ring data per evaluation (numba_healpy.py:73-114) and
 * cache spin-2 angles per sample (tod_bilinear.py:151-199). */
size_t todgpu_ring_table_bytes(int64_t nside);
int todgpu_ring_table_build(int64_t nside, double reach, void *table, size_t bytes, void *stream);

/* Pack a planar (C, N) float32/float64 map (row stride `stride` elements) into
 * N records of 4 components: packed_dtype TODGPU_PACKED_F32 (16 B/pixel, `out`
 * 16-byte aligned), TODGPU_PACKED_BF16 (8 B/pixel, round to nearest even) or
 * TODGPU_PACKED_F64 (32 B/pixel, exact, `out` 16-byte aligned).  No counterpart in the reference, which
 * reads planar mp_stacked (gridint.py:447-450). */
int todgpu_pack_map(const void *planar, int32_t planar_dtype, int64_t C, int64_t N, int64_t stride,
                    int32_t packed_dtype, void *out, void *stream);

/* Spherical-harmonic synthesis of one real RING map component (healpy
 * alm2map stand-in for seeded synthetic skies; the reference's benchmark
 * skies come from healpy.synfast, which is not available here): alm is a
 * device array of (lmax+1)(lmax+2)/2 complex float64 (re, im) pairs in m-major
 * order (index m (2 lmax + 1 - m)/2 + l); map[comp * map_stride + p] receives
 * the value at pixel p.  workspace: todgpu_alm2map_workspace_bytes(nside, lmax)
 * bytes of device memory, overwritten. */
size_t todgpu_alm2map_workspace_bytes(int64_t nside, int32_t lmax);
int todgpu_alm2map(int64_t nside, int32_t lmax, const void *alm, void *workspace, size_t ws_bytes,
                   double *map, int64_t map_stride, int32_t comp, void *stream);

/* FP64 pipe throughput probe (measurement helper; no counterpart in the
 * reference): launches `blocks` CTAs of 256 threads running `iters` rounds of
 * 8 independent FMA chains; *flops receives the floating-point operation count
 * of the launch (host).  `sink` is a device buffer of `blocks` doubles that is
 * never written in practice.  Time it with CUDA events on `stream`. */
int todgpu_fp64_probe(int64_t blocks, int32_t iters, double *sink, double *flops, void *stream);

/* L2 bandwidth probe (measurement helper; no counterpart in the reference):
 * `blocks` CTAs of 256 threads read the device buffer `buf` (16-byte aligned;
 * size it to fit in L2) `iters` times with 16-byte loads that bypass L1;
 * *bytes_read receives the bytes the launch reads (host).  `sink` is a device
 * buffer of `blocks` unsigned ints, never written in practice.  Time it with
 * CUDA events on `stream`. */
int todgpu_l2_probe(const void *buf, size_t bytes, int32_t iters, unsigned *sink, int64_t blocks, double *bytes_read,
                    void *stream);

/*
 * Learned far-sidelobe tail (no counterpart in the reference, whose only
 * tail reduction is the k-means clustering of beam_cluster.py:215-397; the
 * main lobe keeps going through todgpu_gather_accum).  A Fourier-feature MLP
 * maps the pointing to the tail's I/Q/U TOD contribution:
 *   x = (sin t cos p, sin t sin p, cos t, cos psi, sin psi, cos 2psi, sin 2psi)
 *   f = [cos(2 pi freq x), sin(2 pi freq x)]        freq: (n_freq, 7) float32
 *   a_1 = silu(W_0 f + b_0), a_{l+1} = silu(W_l a_l + b_l), y = W_D a_D + b_D
 * with W_0 (width, 2 n_freq), W_l (width, width) for l = 1..depth-1, W_D
 * (n_out, width).  `params` is the flat float32 parameter vector, per layer
 * W then b (todgpu_mlp_param_offsets); `params_bf16` its bfloat16 copy, which
 * the contractions read (float32 accumulation) -- refresh it with
 * todgpu_mlp_sync_bf16 after writing `params`; the Adam step keeps both.
 * Constraints: n_freq a multiple of 64, width a multiple of 128, depth in
 * [1, 8], n_out in [1, 4]; batch row counts (`rows`, `batch`, `chunk`) are
 * multiples of 128.  Workspaces are device memory of
 * todgpu_mlp_workspace_bytes(net, rows) bytes, overwritten.
 */
typedef struct todgpu_mlp {
  int32_t n_freq, width, depth, n_out;
  const float *freq;         /* (n_freq, 7), device */
  float *params;             /* flat float32, device */
  void *params_bf16;         /* flat bfloat16, device */
  float *grad;               /* flat float32 (training only) */
  float *adam_m, *adam_v;    /* flat float32 Adam moments (training only) */
} todgpu_mlp;

/* Forward product of the hidden layers: TODGPU_MLP_TCGEN05 (default: 5th-
 * generation tensor cores, float32 accumulators in tensor memory; widths 128
 * and 256) or TODGPU_MLP_MMA_SYNC (warp-level tensor-core instructions; any
 * width, and the path the backward products always take).  Process-wide;
 * returns the previous setting.  todgpu_mlp_wait_timeouts: number of bounded
 * waits in the tcgen05 kernel that ran out since load (0 in a healthy run;
 * reading it synchronises the device), -1 on a CUDA error. */
#define TODGPU_MLP_TCGEN05 0
#define TODGPU_MLP_MMA_SYNC 1
int todgpu_mlp_set_forward_path(int32_t path);
int64_t todgpu_mlp_wait_timeouts(void);
/* Number of forward layers launched on the tcgen05 path since load (a layer
 * whose shape or tensor maps do not suit it runs on mma.sync instead). */
int64_t todgpu_mlp_tcgen05_launches(void);

int64_t todgpu_mlp_param_count(const todgpu_mlp *net);
/* w_off[l], b_off[l] for l = 0..depth (depth = the head). */
int todgpu_mlp_param_offsets(const todgpu_mlp *net, int64_t *w_off, int64_t *b_off);
size_t todgpu_mlp_workspace_bytes(const todgpu_mlp *net, int64_t rows);
/* Byte offsets of the workspace regions: inputs (rows, 7) f32, features
 * (rows, 2 n_freq) bf16, pre-activations (depth, rows, width) f32,
 * activations (depth, rows, width) bf16, head output / its gradient (rows,
 * n_out) f32, two (rows, width) bf16 gradient buffers, split partial sums,
 * per-row loss; offsets[8] = total bytes. */
int todgpu_mlp_workspace_offsets(const todgpu_mlp *net, int64_t rows, int64_t *offsets);
int todgpu_mlp_sync_bf16(const todgpu_mlp *net, void *stream);
/* x (rows, 7) float32 from n pointings theta, phi, psi (angles_dtype
 * TODGPU_F32 or TODGPU_F64); rows n..rows-1 are zeroed. */
int todgpu_mlp_inputs(const void *theta, const void *phi, const void *psi, int32_t angles_dtype, int64_t n,
                      int64_t rows, float *x, void *stream);
/* y (rows, n_out) float32 = network(x). */
int todgpu_mlp_forward(const todgpu_mlp *net, const float *x, int64_t rows, void *ws, size_t ws_bytes, float *y,
                       void *stream);
/* Mean squared error over the batch against target (rows, n_out) into *loss
 * (device float, optional) and its gradient into net->grad (overwritten). */
int todgpu_mlp_loss_grad(const todgpu_mlp *net, const float *x, const float *target, int64_t rows, void *ws,
                         size_t ws_bytes, float *loss, void *stream);
/* One Adam step (step counts from 1) from net->grad. */
int todgpu_mlp_adam(const todgpu_mlp *net, int64_t step, float lr, float beta1, float beta2, float eps,
                    void *stream);
/* Steps first_step .. first_step+n_steps-1 of Adam (0.9, 0.999, 1e-8) on
 * consecutive batches of `batch` rows of (x, target) (n_rows a multiple of
 * batch, batches taken cyclically), learning rate lr_min + (lr_max - lr_min)
 * (1 + cos(pi step / total_steps)) / 2; loss_per_step (device, n_steps
 * floats, optional) receives each step's loss. */
int todgpu_mlp_train(const todgpu_mlp *net, const float *x, const float *target, int64_t n_rows, int64_t batch,
                     int64_t first_step, int64_t n_steps, int64_t total_steps, float lr_max, float lr_min, void *ws,
                     size_t ws_bytes, float *loss_per_step, void *stream);
/* tod[rows[o] * tod_stride + b] += y_o(theta_b, phi_b, psi_b) scale[o] + shift[o]
 * for b < B, evaluated in chunks of `chunk` samples (rows, scale, shift: host
 * arrays of n_out entries). */
int todgpu_tail_accumulate(const todgpu_mlp *net, const void *theta, const void *phi, const void *psi,
                           int32_t angles_dtype, int64_t B, const int32_t *rows, const double *scale,
                           const double *shift, double *tod, int64_t tod_stride, int64_t chunk, void *ws,
                           size_t ws_bytes, void *stream);

/*
 * Weighted spherical k-means of beam pixels (the clustering of
 * beam_cluster.py:70-188, used by cluster_beam_pixels :215-397).  vec (S, 3)
 * float64 unit vectors and w (S,) float64 weights are device arrays; S < 2^31,
 * 1 <= K <= 8192 clusters.  Workspaces: todgpu_kmeans_workspace_bytes(S, K)
 * bytes of device memory, overwritten.
 *
 * todgpu_kmeans_seed: k-means++ seeding (beam_cluster.py:70-112).  Centroid k
 * is pixel i, the first index with cumsum(p)_i / sum(p) > uniforms[k] (a host
 * array of K draws in [0, 1), the caller's random stream), p_i = w_i for
 * k = 0 and w_i max(1 - max_{j<k} v_i . c_j, 0)^2 after that (w when all
 * p_i are 0).  centroids (K, 3) and chosen (K,) int64 are device outputs.
 * todgpu_kmeans_assign: labels[i] = argmax_k v_i . c_k (first maximum),
 * best[i] = the maximum, with v . c = fma(v2, c2, fma(v1, c1, v0 c0)).
 * todgpu_kmeans_sums: sums (K, 4) = per cluster (sum w x, sum w y, sum w z,
 * sum w), each taken in increasing pixel order (as numpy.bincount does).
 * todgpu_kmeans_argmin: first index of the minimum of best (S,) into *index
 * (device int64).
 */
size_t todgpu_kmeans_workspace_bytes(int64_t S, int32_t K);
int todgpu_kmeans_seed(const double *vec, const double *w, int64_t S, int32_t K, const double *uniforms,
                       double *centroids, int64_t *chosen, void *ws, size_t ws_bytes, void *stream);
int todgpu_kmeans_assign(const double *vec, int64_t S, const double *centroids, int32_t K, int32_t *labels,
                         double *best, void *stream);
int todgpu_kmeans_sums(const double *vec, const double *w, const int32_t *labels, int64_t S, int32_t K,
                       double *sums, void *ws, size_t ws_bytes, void *stream);
int todgpu_kmeans_argmin(const double *best, int64_t S, int64_t *index, void *stream);

/* Library introspection. */
int todgpu_abi_version(void);
const char *todgpu_last_error_string(void);

#ifdef __cplusplus
}
#endif

#endif /* TODGPU_H */
