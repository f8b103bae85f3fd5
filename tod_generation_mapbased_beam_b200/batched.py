"""Batched detectors in one persistent launch (e.g. 64 detectors, each with its
own beam and a scan of its own length).

:class:`DetectorBatch` holds, on the GPU, every detector's beam (vectors and
weights), its scan angles and its (C, n) float64 output, and runs them all
with one ``todgpu_gather_accum_batched`` launch -- the rotation of each sample
derived on the device from its angles (FP64): by default first into float64
parameter buffers, one ``todgpu_pointing_params`` launch per detector, which
the batched gather then reads (``precompute=False``: inside the gather, same
result bit for bit).  The launches are captured in a
CUDA graph on first use and replayed afterwards (``graph=True``), and its
tile size (samples per work tile) is chosen by :mod:`autotune` unless given.

The reference has no batched mode: it loops over beam entries per batch
(sample_based_tod_generation_gridint.py:284-296); one DetectorBatch run equals
one gather per detector (tests/test_gpu_batched.py checks bit-identity).
"""

from __future__ import annotations


import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle, to_device
from .kernels import (_map_tensor, _ncomp, _row_stride, _set_map, beam_order, beam_reach, pointing_buffers,
                      pointing_params, ring_table, table_slots_for)


class DetectorBatch:
    def __init__(self, nside, mp, detectors, comp_indices=(0, 1, 2), interp_mode="bilinear",
                 tile=None, graph=True, tables=True, precompute=True, wide_ctas=False):
        require_cuda()
        if interp_mode not in ("bilinear", "nearest"):
            raise ValueError(f"interp_mode {interp_mode!r} not available on main branch; "
                             "switch to the 'gaussian' or 'bicubic' branch")
        self.nside = int(nside)
        self.interp = _native.BILINEAR if interp_mode == "bilinear" else _native.NEAREST
        self.map = _map_tensor(mp)
        self.C = _ncomp(self.map)
        comps = list(comp_indices)
        if len(comps) != self.C:
            raise ValueError("comp_indices must name one Stokes component per map component")
        self.c_q = comps.index(1) if 1 in comps else -1
        self.c_u = comps.index(2) if 2 in comps else -1
        dev = torch.device("cuda", torch.cuda.current_device())
        self.vec, self.beam, self.angles, self.out, self.centers = [], [], [], [], []
        self.tables = []
        for d in detectors:
            # pixels in the gather's preferred order (neighbours on the sky next to
            # each other; only the order of the pixel sums changes)
            order = torch.from_numpy(beam_order(d["vec_orig"])).to(dev)
            vec = to_device(d["vec_orig"], np.float64).reshape(-1, 3)[order].contiguous()
            self.vec.append(vec)
            self.beam.append(to_device(d["beam_vals"], np.float32).reshape(-1)[order].contiguous())
            ang = [to_device(d[k], np.float32).reshape(-1) for k in ("theta", "phi", "psi")]
            self.angles.append(ang)
            self.out.append(torch.zeros((self.C, ang[0].shape[0]), dtype=torch.float64, device=dev))
            self.centers.append(tuple(d.get("center", (0.0, 0.0))))
            # each detector's own ring table, sized for its own beam: the per-sample
            # spin-2 tables fill every window ring's reserved slots, so a table
            # sized for the widest beam of the batch costs the narrower ones work
            # (tables are cached per reach and shared between equal beams)
            reach = beam_reach(vec, self.nside) if (tables and vec.shape[0]) else 0.0
            self.tables.append(ring_table(self.nside, reach, dev) if reach > 0 else None)
        self.rot = [pointing_buffers(a[0].shape[0], dev) for a in self.angles] if precompute else None
        # wide_ctas: 256-thread CTAs even where the tables fit 128-thread ones
        # (same TOD; for timing and tests)
        self.flags = (0 if tables else _native.FLAG_NO_TABLES) | (_native.FLAG_WIDE_CTAS if wide_ctas else 0)
        self._args = self._make_args()
        self.tile = int(tile) if tile else None
        self.use_graph = graph
        self._graph = None

    @property
    def n_samples(self):
        return sum(a[0].shape[0] for a in self.angles)

    @property
    def n_evals(self):
        return sum(a[0].shape[0] * v.shape[0] for a, v in zip(self.angles, self.vec))

    def _make_args(self):
        arr = (_native.GatherArgs * len(self.vec))()
        for j, (vec, bv, ang, out, cen) in enumerate(zip(self.vec, self.beam, self.angles, self.out,
                                                          self.centers)):
            a = arr[j]
            a.abi_version = _native.ABI_VERSION
            a.interp = self.interp
            a.nside = self.nside
            a.B = ang[0].shape[0]
            a.S = vec.shape[0]
            a.C = self.C
            a.c_q, a.c_u = self.c_q, self.c_u
            _set_map(a, self.map)
            a.vec_orig = vec.data_ptr()
            if self.rot is not None:
                a.params_dtype = _native.F64
                (a.axes, a.cos_a, a.sin_a, a.ax_pts, a.cos_p, a.sin_p) = (t.data_ptr() for t in self.rot[j])
            else:
                a.params_dtype = _native.ANGLES
                a.theta, a.phi, a.psi = (t.data_ptr() for t in ang)
                a.angles_dtype = _native.F32
                a.center_phi, a.center_theta = cen
            a.beam_vals = bv.data_ptr()
            a.tod = out.data_ptr()
            a.tod_stride = _row_stride(out)
            a.flags = self.flags
            a.ring_table = None if self.tables[j] is None else self.tables[j].data_ptr()
            a.tab_slots = table_slots_for(self.tables[j], self.nside)
        return arr

    def truncated(self, fraction):
        """A batch over the first ``fraction`` of every detector's samples that
        shares this batch's device buffers (a cheaper stand-in with the same
        detectors and the same proportions, e.g. for timing tile sizes)."""
        import copy

        b = copy.copy(self)
        b.angles = [[t[:max(1, int(t.shape[0] * fraction))] for t in ang] for ang in self.angles]
        b.out = [o[:, :a[0].shape[0]] for o, a in zip(self.out, b.angles)]
        b._args = b._make_args()
        b._graph = None
        b.tile = None
        return b

    def launch(self, tile=None):
        """Zero the outputs and launch once on the current stream (no graph)."""
        for o in self.out:
            o.zero_()
        if self.rot is not None:
            for ang, rot, cen in zip(self.angles, self.rot, self.centers):
                pointing_params(*ang, cen[0], cen[1], out=rot)
        t = int(tile or self.tile or 256)
        _native.check(_native.lib().todgpu_gather_accum_batched(self._args, len(self._args), t,
                                                                stream_handle()))

    def run(self):
        """All detectors' (C, n) float64 outputs (CUDA tensors, in order)."""
        if self.tile is None:
            from .autotune import choose_tile

            self.tile = choose_tile(self)
        if not self.use_graph:
            self.launch()
            return self.out
        if self._graph is None:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):
                self.launch()  # first launch configures the kernel outside the capture
            torch.cuda.current_stream().wait_stream(side)
            self._graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self._graph):
                self.launch()
        self._graph.replay()
        return self.out

    def release(self):
        self._graph = None
