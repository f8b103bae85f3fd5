"""Streaming day driver: the GPU counterpart of the reference's day loop.

Reference: ``tod_exact_gen_batched`` and ``_process_day``
(sample_based_tod_generation_gridint.py:208-333) with the scan IO of
tod_io.py:39-143.  One day of scan samples -- ``theta_N.npy``, ``phi_N.npy``,
``psi_N.npy`` in a scan folder -- becomes ``tod_day`` of shape (3, n), float64,
axis 0 the Stokes component [I, Q, U], saved as ``tod_day_N.npy``; every beam
entry's contribution is added into the components it carries
(gridint.py:283-298).

Two pointing modes:

* ``"reference"``: per batch, the reference's host preparation
  (``precompute_rotation_vector_batch`` on float32 angles, psi - beta) and the
  drop-in ``beam_tod_batch``; each entry's float32 result is added into the
  float64 day array exactly as the reference driver does.  Bit-level parity
  with the reference (kernel tolerance 1e-12, then the same float32 casts).
* ``"device"`` (default): the scan is streamed through pinned host buffers in
  chunks; a copy stream uploads chunk i+1 while the compute stream runs chunk
  i (rotation derived on the GPU in float64 from the angles, no float32
  parameter rounding) and a third stream downloads chunk i-1.  Entries are
  accumulated in float64 on the device.
"""

from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native
from ._device import require_cuda
from .kernels import beam_center_angles, gather_accum_angles
from .tod_core import _INTERP, beam_tod_batch, component_slots, device_beam, device_map
from .tod_rotations import precompute_rotation_vector_batch

__all__ = ["load_scan_information", "open_scan_day", "DayRunner", "tod_exact_gen_batched",
           "process_day", "prepare_beam_data", "load_sky"]


def load_sky(path_to_map):
    """The sky as the reference's main loads it (gridint.py:406-408): fields
    0, 1, 2 of a HEALPix FITS map, RING order, each cast to float32."""
    from .map_io import read_map

    return [m.astype(np.float32) for m in read_map(path_to_map, field=(0, 1, 2))]


def prepare_beam_data(beam_filenames, folder_beam=None, thresholds=None, config=None):
    """Drop-in for ``prepare_beam_data`` (gridint.py:92-159): one entry per
    distinct beam file, keyed by file name, with ``ra, dec`` (offset grids as
    ``load_beam`` binds them), ``beam_vals`` (float32, normalised by their sum
    unless it is 0), ``sel`` (``10 log10(|b| + 1e-30) > dB cut`` for the
    file's power threshold), ``comp_indices`` (the Stokes components sharing
    the file, in order), ``n_sel`` and ``vec_orig`` (float32 (S, 3): theta =
    pi/2 - dec, longitude ra).

    ``folder_beam`` and ``thresholds`` ({file name: power fraction}) default to
    a :class:`tod_config.TodConfig`'s FOLDER_BEAM and its I, Q, U thresholds
    (a file named for several components takes the last one, as the
    reference's dictionary does)."""
    from .map_io import load_beam
    from .workloads import compute_db_threshold_from_power

    if config is not None:
        folder_beam = config.FOLDER_BEAM if folder_beam is None else folder_beam
        if thresholds is None:
            thresholds = {config.beam_file_I: config.power_threshold_I,
                          config.beam_file_Q: config.power_threshold_Q,
                          config.beam_file_U: config.power_threshold_U}
    if folder_beam is None or thresholds is None:
        raise ValueError("give folder_beam and thresholds, or a config")
    groups = {}
    for i, bf in enumerate(beam_filenames):
        groups.setdefault(bf, []).append(i)
    beam_data = {}
    for bf, comp_indices in groups.items():
        ra, dec, pixel_map = load_beam(folder_beam, bf)
        db_cut = compute_db_threshold_from_power(pixel_map, thresholds[bf])
        with np.errstate(divide="ignore", invalid="ignore"):
            sel = 10 * np.log10(np.abs(pixel_map) + 1e-30) > db_cut
        beam_vals = pixel_map[sel].astype(np.float32)
        norm = beam_vals.sum()
        if norm != 0:
            beam_vals /= norm
        theta_orig = np.pi / 2 - dec
        vec_orig = np.stack([np.sin(theta_orig) * np.cos(ra), np.sin(theta_orig) * np.sin(ra),
                             np.cos(theta_orig)], axis=-1)[sel].astype(np.float32)
        beam_data[bf] = {"ra": ra, "dec": dec, "beam_vals": beam_vals, "sel": sel,
                         "comp_indices": comp_indices, "n_sel": int(sel.sum()), "vec_orig": vec_orig}
    return beam_data


def load_scan_information(folder):
    """(number of days, sample rate) from the ``psi_N.npy`` files of a scan
    folder (tod_io.py:39-67)."""
    files = [f for f in os.listdir(folder) if f.startswith("psi")]
    if not files:
        raise FileNotFoundError(f"No 'psi_*.npy' files found in scan folder {folder!r}")
    try:
        max_index = max(int(f.split("_")[1].split(".")[0]) for f in files)
    except (IndexError, ValueError) as exc:
        raise ValueError(f"Could not parse scan-file index from filenames in {folder!r}. "
                         f"Expected names like 'psi_<N>.npy', got: {files[:5]!r}") from exc
    fsamp = np.load(os.path.join(folder, files[0]), mmap_mode="r").shape[0] / 86400
    return max_index + 1, fsamp


def open_scan_day(folder_scan, day_index):
    """Memory-mapped (theta, phi, psi) of one day (tod_io.py:70-95)."""
    return tuple(np.load(os.path.join(folder_scan, f"{name}_{day_index}.npy"), mmap_mode="r")
                 for name in ("theta", "phi", "psi"))


def _rows(C, comps):
    """(first row, row step) when comps is an arithmetic progression with a
    positive step, else None."""
    if C == 1:
        return comps[0], 1
    step = comps[1] - comps[0]
    if step <= 0 or any(comps[i + 1] - comps[i] != step for i in range(C - 1)):
        return None
    return comps[0], step


@dataclass
class _Entry:
    comps: list
    c_q: int
    c_u: int
    vec: torch.Tensor
    beam: torch.Tensor
    mp: torch.Tensor
    center: tuple
    rows: tuple | None


@dataclass
class DayRunner:
    """Computes (3, n) float64 day TOD for a set of beam entries.

    ``beam_data`` is the reference's dict of beam entries (``vec_orig``,
    ``beam_vals``, ``comp_indices``, ``mp_stacked``, ``ra``, ``dec``); ``mp``
    the [I, Q, U] map list used when an entry has no ``mp_stacked``."""

    beam_data: dict
    nside: int
    mp: list | None = None
    interp_mode: str = "bilinear"
    chunk: int = 1 << 20
    pointing: str = "device"
    _entries: list = field(default_factory=list, init=False)

    def __post_init__(self):
        if self.interp_mode not in _INTERP:
            raise ValueError(f"interp_mode {self.interp_mode!r} not available on main branch; "
                             "switch to the 'gaussian' or 'bicubic' branch")
        if self.pointing not in ("device", "reference"):
            raise ValueError("pointing must be 'device' or 'reference'")
        require_cuda()
        if self.pointing == "device":
            for data in self.beam_data.values():
                comps = list(data["comp_indices"])
                c_q, c_u = component_slots(comps)
                vec, bv = device_beam(data["vec_orig"], data["beam_vals"], torch.float64)
                self._entries.append(_Entry(
                    comps, c_q, c_u, vec, bv, device_map(data, self.mp),
                    beam_center_angles(data["ra"], data["dec"]), _rows(len(comps), comps)))

    # -- reference pointing -------------------------------------------------
    def _run_reference(self, theta, phi, psi):
        n = len(phi)
        first = next(iter(self.beam_data.values()))
        ra0, dec0 = first["ra"], first["dec"]
        tod_day = np.zeros((3, n))
        bs = max(1, min(self.chunk, n))
        for s0 in range(0, n, bs):
            s1 = min(s0 + bs, n)
            th = np.array(theta[s0:s1], dtype=np.float32)
            ph = np.array(phi[s0:s1], dtype=np.float32)
            ps = np.array(psi[s0:s1], dtype=np.float32)
            rot, beta = precompute_rotation_vector_batch(ra0, dec0, ph, th)
            psis = -beta + ps
            batch = np.zeros((3, s1 - s0))
            for data in self.beam_data.values():
                contrib = beam_tod_batch(self.nside, self.mp, data, rot, ph, th, psis,
                                         interp_mode=self.interp_mode)
                for comp, vals in contrib.items():
                    batch[comp] += vals
            tod_day[:, s0:s1] = batch
        return tod_day

    # -- device pointing ----------------------------------------------------
    def _accumulate(self, th, ph, ps, out):
        interp = _INTERP[self.interp_mode]
        for e in self._entries:
            C = len(e.comps)
            if e.rows is not None:
                r0, step = e.rows
                dst = out[r0:r0 + (C - 1) * step + 1:step]
                gather_accum_angles(interp, e.vec, th, ph, ps, e.center[0], e.center[1], self.nside,
                                    e.mp, e.beam, dst, e.c_q, e.c_u)
            else:
                tmp = torch.zeros((C, out.shape[1]), dtype=torch.float64, device=out.device)
                gather_accum_angles(interp, e.vec, th, ph, ps, e.center[0], e.center[1], self.nside,
                                    e.mp, e.beam, tmp, e.c_q, e.c_u)
                out.index_add_(0, torch.tensor(e.comps, device=out.device), tmp)

    def _run_device(self, theta, phi, psi):
        n = len(phi)
        dev = torch.device("cuda", torch.cuda.current_device())
        tod_day = np.empty((3, n))
        if n == 0:
            return tod_day
        ch = max(1, min(self.chunk, n))
        pin_in = [torch.empty((3, ch), dtype=torch.float32, pin_memory=True) for _ in range(2)]
        pin_out = [torch.empty((3, ch), dtype=torch.float64, pin_memory=True) for _ in range(2)]
        d_in = [torch.empty((3, ch), dtype=torch.float32, device=dev) for _ in range(2)]
        d_out = [torch.empty((3, ch), dtype=torch.float64, device=dev) for _ in range(2)]
        compute = torch.cuda.current_stream(dev)
        up = torch.cuda.Stream(dev)
        down = torch.cuda.Stream(dev)
        ev_up = [torch.cuda.Event() for _ in range(2)]
        ev_comp = [torch.cuda.Event() for _ in range(2)]
        ev_down = [None, None]
        pending = [None, None]  # (slice, length) waiting in pin_out[k]

        def drain(k):
            if ev_down[k] is not None:
                ev_down[k].synchronize()
                (s0, m) = pending[k]
                tod_day[:, s0:s0 + m] = pin_out[k].numpy()[:, :m]
                ev_down[k] = None

        for i, s0 in enumerate(range(0, n, ch)):
            k = i & 1
            m = min(ch, n - s0)
            drain(k)  # pin_out[k] and (via the order of events) pin_in[k] are free again
            host = pin_in[k].numpy()
            host[0, :m] = theta[s0:s0 + m]
            host[1, :m] = phi[s0:s0 + m]
            host[2, :m] = psi[s0:s0 + m]
            with torch.cuda.stream(up):
                up.wait_event(ev_comp[k])  # the previous user of d_in[k] has finished
                d_in[k][:, :m].copy_(pin_in[k][:, :m], non_blocking=True)
                ev_up[k].record(up)
            compute.wait_event(ev_up[k])
            out = d_out[k][:, :m]
            out.zero_()
            self._accumulate(d_in[k][0, :m], d_in[k][1, :m], d_in[k][2, :m], out)
            ev_comp[k].record(compute)
            with torch.cuda.stream(down):
                down.wait_event(ev_comp[k])
                pin_out[k][:, :m].copy_(out, non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(down)
            ev_down[k] = ev
            pending[k] = (s0, m)
            # pin_in[k] is reused two chunks later, after drain(k) has waited for
            # this chunk's download, which follows its upload and compute
        for k in range(2):
            drain(k)
        return tod_day

    def run(self, theta, phi, psi):
        """(3, n) float64 TOD of one day for scan arrays theta, phi, psi."""
        if not (len(theta) == len(phi) == len(psi)):
            raise ValueError("theta, phi and psi must have the same length")
        if self.pointing == "reference":
            return self._run_reference(theta, phi, psi)
        return self._run_device(theta, phi, psi)


def tod_exact_gen_batched(beam_data, day_index, mp, batch_size, folder_scan, nside,
                          interp_mode="bilinear", pointing="device"):
    """GPU counterpart of gridint.py:208-305: the (3, n) float64 TOD of one
    day read from ``folder_scan``; ``batch_size`` is the streaming chunk."""
    theta, phi, psi = open_scan_day(folder_scan, day_index)
    runner = DayRunner(beam_data, nside, mp, interp_mode, chunk=batch_size, pointing=pointing)
    return runner.run(theta, phi, psi)


def process_day(day_index, beam_data, mp, batch_size, folder_scan, folder_out, nside,
                interp_mode="bilinear", pointing="device"):
    """gridint.py:311-333: compute one day and save ``tod_day_N.npy``;
    returns (day, ok, error message)."""
    try:
        tod_day = tod_exact_gen_batched(beam_data, day_index, mp, batch_size, folder_scan, nside,
                                        interp_mode, pointing)
        np.save(os.path.join(folder_out, f"tod_day_{day_index}.npy"), tod_day)
        return day_index, True, None
    except (ValueError, RuntimeError, OSError, _native.TodGpuError) as e:
        return day_index, False, str(e)
