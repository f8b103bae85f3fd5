"""Beam-pixel clustering on the GPU: drop-in for the reference module
``beam_cluster`` (beam_cluster.py).

:func:`cluster_beam_pixels` keeps the reference's signature, modes and
outputs (beam_cluster.py:215-397): in full mode all pixels are clustered into
``n_clusters`` centroids; in hybrid mode (``tail_fraction``) the weakest
pixels holding ``tail_fraction`` of the power form the tail and only they are
clustered, the main-lobe pixels pass through unchanged, and the output is
``[main pixels in ascending weight order..., tail centroids...]`` with the
weights renormalised.  :func:`split_main_tail` is that main/tail split on its
own (beam_cluster.py:307-326), which the learned-tail form also uses.

The weighted spherical k-means (beam_cluster.py:70-188) runs in libtodgpu:
k-means++ seeding, the (pixels x clusters) similarity argmax and the
per-cluster sums are GPU kernels; the O(clusters) bookkeeping between
iterations (empty clusters, normalisation, convergence) stays in numpy with
the reference's operations.  The random stream is the reference's
(``numpy.random.default_rng(random_state)``): seeding consumes one uniform per
centroid, as ``Generator.choice`` with probabilities does.  Per-cluster sums
are taken in pixel order like ``numpy.bincount``; the similarities use the
multiply-add order of a BLAS product, and seeding's cumulative sums are
blocked, so a result can differ from the reference's only where two
candidates tie to the last bit.
"""

from __future__ import annotations

import ctypes
import logging
import time

import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle

__all__ = ["cluster_beam_pixels", "split_main_tail"]

log = logging.getLogger(__name__)


def _note(verbose, msg, *args):
    """Progress report of the clustering, on this module's logger (INFO)
    when ``verbose``."""
    if verbose:
        log.info(msg, *args)


def split_main_tail(beam_vals, tail_fraction):
    """(main_idx, tail_idx): pixels sorted by ascending weight; the tail is the
    smallest prefix whose cumulative weight exceeds ``tail_fraction``
    (searchsorted 'right' on the float32 cumulative sum), kept between 1 and
    S - 1 pixels; main_idx ascending in weight (beam_cluster.py:307-326)."""
    bv = np.asarray(beam_vals)
    S = len(bv)
    order = np.argsort(bv)
    cumsum = np.cumsum(bv[order])
    n_tail = int(np.searchsorted(cumsum, tail_fraction, side="right"))
    n_tail = max(1, min(n_tail, S - 1))
    return order[n_tail:], order[:n_tail]


class _GpuKMeans:
    """Device buffers and calls of one clustering problem."""

    def __init__(self, vec, w, K):
        self.dev = require_cuda()
        self.S = int(vec.shape[0])
        self.K = int(K)
        self.vec = torch.from_numpy(np.ascontiguousarray(vec, np.float64)).to(self.dev)
        self.w = torch.from_numpy(np.ascontiguousarray(w, np.float64)).to(self.dev)
        lib = _native.lib()
        nb = int(lib.todgpu_kmeans_workspace_bytes(self.S, self.K))
        if nb == 0:
            raise ValueError(f"unsupported clustering size S={self.S}, K={self.K} (K <= 8192)")
        self.ws = torch.empty(nb, dtype=torch.uint8, device=self.dev)
        self.labels = torch.empty(self.S, dtype=torch.int32, device=self.dev)
        self.best = torch.empty(self.S, dtype=torch.float64, device=self.dev)
        self.sums = torch.empty((self.K, 4), dtype=torch.float64, device=self.dev)
        self.idx = torch.empty(1, dtype=torch.int64, device=self.dev)

    def seed(self, uniforms):
        u = np.ascontiguousarray(uniforms, np.float64)
        cent = torch.empty((self.K, 3), dtype=torch.float64, device=self.dev)
        chosen = torch.empty(self.K, dtype=torch.int64, device=self.dev)
        _native.check(_native.lib().todgpu_kmeans_seed(
            self.vec.data_ptr(), self.w.data_ptr(), self.S, self.K, u.ctypes.data_as(ctypes.c_void_p),
            cent.data_ptr(), chosen.data_ptr(), self.ws.data_ptr(), self.ws.numel(), stream_handle()))
        return cent.cpu().numpy()

    def assign(self, centroids):
        c = torch.from_numpy(np.ascontiguousarray(centroids, np.float64)).to(self.dev)
        _native.check(_native.lib().todgpu_kmeans_assign(self.vec.data_ptr(), self.S, c.data_ptr(), self.K,
                                                         self.labels.data_ptr(), self.best.data_ptr(),
                                                         stream_handle()))

    def cluster_sums(self):
        _native.check(_native.lib().todgpu_kmeans_sums(self.vec.data_ptr(), self.w.data_ptr(),
                                                       self.labels.data_ptr(), self.S, self.K,
                                                       self.sums.data_ptr(), self.ws.data_ptr(), self.ws.numel(),
                                                       stream_handle()))
        return self.sums.cpu().numpy()

    def argmin_best(self):
        _native.check(_native.lib().todgpu_kmeans_argmin(self.best.data_ptr(), self.S, self.idx.data_ptr(),
                                                         stream_handle()))
        return int(self.idx.item())


def _kmeans_sphere(vec, bvals, K, max_iter, tol, rng, label="", verbose=True):
    """Weighted spherical k-means; returns (centroids (K, 3) float64, labels
    (S,) int32), following beam_cluster.py:115-188."""
    km = _GpuKMeans(vec, bvals, K)
    centroids = km.seed([rng.random() for _ in range(K)])
    cos_tol = np.cos(tol)
    cos_disp = np.full(K, -1.0)
    for iteration in range(max_iter):
        km.assign(centroids)
        sums = km.cluster_sums()
        new_centroids = sums[:, :3].copy()
        new_weights = sums[:, 3].copy()
        empty = new_weights == 0
        if empty.any():
            idx = km.argmin_best()
            for k in np.where(empty)[0]:
                new_centroids[k] = vec[idx]
                new_weights[k] = bvals[idx]
        norms = np.linalg.norm(new_centroids, axis=1, keepdims=True)
        norms = np.where(norms > 0, norms, 1.0)
        new_centroids /= norms
        cos_disp = np.clip((centroids * new_centroids).sum(axis=1), -1.0, 1.0)
        centroids = new_centroids
        if cos_disp.min() > cos_tol:
            _note(verbose, "k-means%s: settled after %d iterations (largest centroid move %.3f arcmin)",
                  label, iteration + 1, np.degrees(float(np.arccos(cos_disp).max())) * 60)
            break
    else:
        _note(verbose, "k-means%s: stopped at the iteration limit %d (largest centroid move %.3f arcmin)",
              label, max_iter, np.degrees(float(np.arccos(cos_disp).max())) * 60)
    km.assign(centroids)
    return centroids, km.labels.cpu().numpy().astype(np.int32)


def _spread(vec, centroids, labels, label, verbose):
    if not verbose:
        return
    c = np.clip((vec * centroids[labels]).sum(axis=1), -1.0, 1.0)
    arcmin = np.degrees(np.arccos(c)) * 60.0
    _note(True, "k-means%s: pixel to centroid distance %.2f arcmin on average, %.2f at the 95th percentile, "
          "%.2f at most", label, arcmin.mean(), np.percentile(arcmin, 95), arcmin.max())


def cluster_beam_pixels(vec_orig, beam_vals, n_clusters, tail_fraction=None, max_iter=150, tol=1e-5,
                        random_state=42, verbose=True):
    """(vec_out (K_out, 3) float32, bvals_out (K_out,) float32, labels (S,)
    int32): see the module docstring and beam_cluster.py:215-397."""
    vec_orig = np.asarray(vec_orig)
    beam_vals = np.asarray(beam_vals)
    S = len(beam_vals)
    if tail_fraction is None:
        K = min(n_clusters, S)
        if K >= S:
            return vec_orig.copy(), beam_vals.copy(), np.arange(S, dtype=np.int32)
        t0 = time.time()
        vec = vec_orig.astype(np.float64)
        bvals = beam_vals.astype(np.float64)
        centroids, labels = _kmeans_sphere(vec, bvals, K, max_iter, tol, np.random.default_rng(random_state),
                                           verbose=verbose)
        weights = np.zeros(K, dtype=np.float64)
        np.add.at(weights, labels, bvals)
        weights /= weights.sum()
        _note(verbose, "clustered all %d beam pixels into %d entries in %.2f s", S, K, time.time() - t0)
        _spread(vec, centroids, labels, "", verbose)
        return centroids.astype(np.float32), weights.astype(np.float32), labels

    if not (0.0 < tail_fraction < 1.0):
        raise ValueError(f"tail_fraction must be in (0, 1), got {tail_fraction!r}")
    t0 = time.time()
    main_idx, tail_idx = split_main_tail(beam_vals, tail_fraction)
    n_main, n_tail = len(main_idx), len(tail_idx)
    tp = float(beam_vals[tail_idx].sum())
    _note(verbose, "main lobe: %d pixels kept as they are (%.1f%% of the weight); tail: %d pixels (%.1f%%)",
          n_main, 100 * (1 - tp), n_tail, 100 * tp)
    K_tail = min(n_clusters, n_tail)
    if K_tail >= n_tail:
        vec_tail = vec_orig[tail_idx]
        bv_tail = beam_vals[tail_idx]
        tail_labels = np.arange(n_tail, dtype=np.int32)
        _note(verbose, "tail left unclustered: %d pixels, no more than the %d entries asked for", n_tail,
              n_clusters)
    else:
        vec_t = vec_orig[tail_idx].astype(np.float64)
        bv_t = beam_vals[tail_idx].astype(np.float64)
        centroids_t, tail_labels = _kmeans_sphere(vec_t, bv_t, K_tail, max_iter, tol,
                                                  np.random.default_rng(random_state), label=" tail",
                                                  verbose=verbose)
        cw = np.zeros(K_tail, dtype=np.float64)
        np.add.at(cw, tail_labels, bv_t)
        vec_tail = centroids_t.astype(np.float32)
        bv_tail = cw.astype(np.float32)
        _note(verbose, "tail: %d pixels clustered into %d entries in %.2f s", n_tail, K_tail, time.time() - t0)
        _spread(vec_t, centroids_t, tail_labels, " tail", verbose)
    vec_out = np.concatenate([vec_orig[main_idx], vec_tail], axis=0)
    bv_out = np.concatenate([beam_vals[main_idx], bv_tail], axis=0)
    bv_out = (bv_out / bv_out.sum()).astype(np.float32)
    labels = np.empty(S, dtype=np.int32)
    labels[main_idx] = np.arange(n_main, dtype=np.int32)
    labels[tail_idx] = n_main + tail_labels
    _note(verbose, "beam entry now has %d pixels in place of %d", n_main + K_tail, S)
    return vec_out, bv_out, labels
