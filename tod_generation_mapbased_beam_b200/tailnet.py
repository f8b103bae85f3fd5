"""The learned far-sidelobe tail network (``todgpu_mlp_*`` in libtodgpu).

A Fourier-feature MLP of the pointing -- boresight unit vector and roll psi,
as (sin t cos p, sin t sin p, cos t, cos psi, sin psi, cos 2psi, sin 2psi) --
predicting the I/Q/U TOD contribution of a beam's far sidelobes.  Training
and evaluation run in the library's own kernels: bfloat16 weights and
activations, float32 sums on the tensor cores, float32 master weights and
Adam moments.  :class:`TailNet` owns the device buffers and the target
normalisation (per-output shift and scale, applied on the device when the
prediction is added into a TOD).

The reference has no learned tail; its tail reduction is the k-means
clustering of beam_cluster.py:215-397, whose main/tail split
``beam_cluster.split_main_tail`` reproduces.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _native
from ._device import require_cuda, stream_handle

ROW_ALIGN = 128  # batch row counts are multiples of this


def _pad(n):
    return max(ROW_ALIGN, (int(n) + ROW_ALIGN - 1) // ROW_ALIGN * ROW_ALIGN)


class TailNet:
    """Fourier-feature MLP on the GPU.

    ``n_freq`` random frequencies (2 n_freq features), ``depth`` SiLU layers of
    ``width`` units, ``n_out`` outputs.  Frequencies are drawn N(0, sigma^2)
    with ``sigma = (sigma_dir, sigma_psi)`` for the three direction inputs and
    the four roll inputs (in cycles per unit of input)."""

    def __init__(self, n_freq=256, width=256, depth=4, n_out=3, sigma=(1.0, 0.5), seed=0, device=None):
        self.device = device if device is not None else require_cuda()
        self.dims = (int(n_freq), int(width), int(depth), int(n_out))
        self.sigma = tuple(float(s) for s in sigma)
        self.seed = int(seed)
        rng = np.random.default_rng(seed)
        F, H, D, O = self.dims
        freq = np.empty((F, 7), np.float32)
        freq[:, :3] = rng.standard_normal((F, 3)) * self.sigma[0]
        freq[:, 3:] = rng.standard_normal((F, 4)) * self.sigma[1]
        self.freq = torch.from_numpy(freq).to(self.device)
        self.desc = _native.MlpDesc()
        self.desc.n_freq, self.desc.width, self.desc.depth, self.desc.n_out = F, H, D, O
        lib = _native.lib()
        n = int(lib.todgpu_mlp_param_count(ctypes.byref(self.desc)))
        if n < 0:
            raise ValueError(f"unsupported network shape {self.dims}: " + lib.todgpu_last_error_string().decode())
        self.n_params = n
        w_off = (ctypes.c_int64 * (D + 1))()
        b_off = (ctypes.c_int64 * (D + 1))()
        _native.check(lib.todgpu_mlp_param_offsets(ctypes.byref(self.desc), w_off, b_off))
        self.w_off, self.b_off = list(w_off), list(b_off)
        p = np.zeros(n, np.float32)
        for l in range(D + 1):  # uniform +-sqrt(6 / fan_in) (He), small head
            fan_in = 2 * F if l == 0 else H
            n_out_l = H if l < D else O
            bound = np.sqrt(6.0 / fan_in) * (1.0 if l < D else 0.1)
            p[self.w_off[l]:self.w_off[l] + n_out_l * fan_in] = rng.uniform(-bound, bound, n_out_l * fan_in)
        self.params = torch.from_numpy(p).to(self.device)
        self.params_bf16 = torch.empty(n, dtype=torch.bfloat16, device=self.device)
        self.grad = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.adam_m = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.adam_v = torch.zeros(n, dtype=torch.float32, device=self.device)
        self.step = 0
        self.shift = np.zeros(O)
        self.scale = np.ones(O)
        self._ws = {}
        self._bind()
        self.sync_bf16()

    # -- buffers ------------------------------------------------------------
    def _bind(self):
        d = self.desc
        d.freq = self.freq.data_ptr()
        d.params = self.params.data_ptr()
        d.params_bf16 = self.params_bf16.data_ptr()
        d.grad = self.grad.data_ptr()
        d.adam_m = self.adam_m.data_ptr()
        d.adam_v = self.adam_v.data_ptr()

    def sync_bf16(self):
        """Refresh the bfloat16 copy after the float32 parameters changed."""
        _native.check(_native.lib().todgpu_mlp_sync_bf16(ctypes.byref(self.desc), stream_handle()))

    def workspace(self, rows):
        rows = int(rows)
        ws = self._ws.get(rows)
        if ws is None:
            nbytes = int(_native.lib().todgpu_mlp_workspace_bytes(ctypes.byref(self.desc), rows))
            if nbytes == 0:
                raise ValueError(f"rows must be a positive multiple of {ROW_ALIGN}, got {rows}")
            ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._ws[rows] = ws
        return ws

    def ws_region(self, rows, name):
        """Raw view of one workspace region (see MLP_WS_REGIONS) of the
        ``rows``-row workspace, as a uint8 tensor."""
        off = (ctypes.c_int64 * (len(_native.MLP_WS_REGIONS) + 1))()
        _native.check(_native.lib().todgpu_mlp_workspace_offsets(ctypes.byref(self.desc), int(rows), off))
        i = _native.MLP_WS_REGIONS.index(name)
        return self.workspace(rows)[off[i]:off[i + 1]]

    def layer(self, l):
        """(W, b) float32 views of layer l (l = depth is the head)."""
        F, H, D, O = self.dims
        n_out = H if l < D else O
        n_in = (2 * F if l == 0 else H) if l < D else H
        W = self.params[self.w_off[l]:self.w_off[l] + n_out * n_in].view(n_out, n_in)
        return W, self.params[self.b_off[l]:self.b_off[l] + n_out]

    # -- inputs -------------------------------------------------------------
    def _angles(self, theta, phi, psi):
        th = torch.as_tensor(theta, device=self.device)
        if th.dtype not in (torch.float32, torch.float64):
            th = th.double()
        ph = torch.as_tensor(phi, device=self.device, dtype=th.dtype).contiguous()
        ps = torch.as_tensor(psi, device=self.device, dtype=th.dtype).contiguous()
        th = th.contiguous()
        if ph.numel() != th.numel() or ps.numel() != th.numel():
            raise ValueError("theta, phi and psi must have the same length")
        return th, ph, ps

    def inputs(self, theta, phi, psi, rows=None):
        """(rows, 7) float32 inputs of the pointings (rows padded to 128)."""
        th, ph, ps = self._angles(theta, phi, psi)
        n = th.numel()
        rows = _pad(n) if rows is None else int(rows)
        x = torch.empty((rows, 7), dtype=torch.float32, device=self.device)
        dt = _native.F32 if th.dtype == torch.float32 else _native.F64
        _native.check(_native.lib().todgpu_mlp_inputs(th.data_ptr(), ph.data_ptr(), ps.data_ptr(), dt, n, rows,
                                                      x.data_ptr(), stream_handle()))
        return x

    # -- evaluation and training -------------------------------------------
    def forward(self, x):
        """Raw network output (rows, n_out) float32 for inputs x (rows, 7)."""
        x = x.contiguous()
        rows = x.shape[0]
        ws = self.workspace(rows)
        y = torch.empty((rows, self.dims[3]), dtype=torch.float32, device=self.device)
        _native.check(_native.lib().todgpu_mlp_forward(ctypes.byref(self.desc), x.data_ptr(), rows, ws.data_ptr(),
                                                       ws.numel(), y.data_ptr(), stream_handle()))
        return y

    def loss_grad(self, x, target):
        """Mean squared error of one batch (float) and its gradient (the
        network's ``grad`` tensor, overwritten)."""
        x, target = x.contiguous(), target.contiguous()
        rows = x.shape[0]
        ws = self.workspace(rows)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        _native.check(_native.lib().todgpu_mlp_loss_grad(ctypes.byref(self.desc), x.data_ptr(), target.data_ptr(),
                                                         rows, ws.data_ptr(), ws.numel(), loss.data_ptr(),
                                                         stream_handle()))
        return float(loss.item()), self.grad

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        _native.check(_native.lib().todgpu_mlp_adam(ctypes.byref(self.desc), self.step, lr, beta1, beta2, eps,
                                                    stream_handle()))

    def set_normalisation(self, target):
        """Per-output shift (mean) and scale (standard deviation) of float64
        targets (n, n_out); training sees (target - shift) / scale."""
        t = np.asarray(target, np.float64)
        self.shift = t.mean(0)
        sd = t.std(0)
        self.scale = np.where(sd > 0, sd, 1.0)

    def fit(self, x, target, steps, batch=8192, lr_max=2e-3, lr_min=2e-5, chunk_steps=500):
        """Adam on (x, target): ``x`` (n, 7) float32 CUDA inputs, ``target``
        (n, n_out) float64 (host or device) in physical units; n is trimmed
        to a multiple of ``batch``.  Sets the normalisation from the targets.
        Returns the per-step losses (normalised units)."""
        batch = _pad(batch)
        t = target.detach().cpu().numpy() if isinstance(target, torch.Tensor) else np.asarray(target)
        n = (x.shape[0] // batch) * batch
        if n == 0:
            raise ValueError(f"need at least {batch} training rows")
        self.set_normalisation(t[:n])
        tn = torch.from_numpy(((t[:n] - self.shift) / self.scale).astype(np.float32)).to(self.device)
        xs = x[:n].contiguous()
        ws = self.workspace(batch)
        steps = int(steps)
        losses = torch.empty(max(steps, 1), dtype=torch.float32, device=self.device)
        lib = _native.lib()
        s0 = self.step
        done = 0
        while done < steps:
            k = min(chunk_steps, steps - done)
            _native.check(lib.todgpu_mlp_train(ctypes.byref(self.desc), xs.data_ptr(), tn.data_ptr(), n, batch,
                                               s0 + done, k, s0 + steps, lr_max, lr_min, ws.data_ptr(), ws.numel(),
                                               losses[done:].data_ptr(), stream_handle()))
            done += k
        self.step = s0 + steps
        return losses[:steps].cpu().numpy()

    def predict(self, theta, phi, psi):
        """(n, n_out) float64 prediction in physical units."""
        n = int(torch.as_tensor(theta).numel())
        y = self.forward(self.inputs(theta, phi, psi))[:n].double().cpu().numpy()
        return y * self.scale + self.shift

    def accumulate(self, theta, phi, psi, tod, rows=(0, 1, 2), chunk=1 << 20):
        """tod[rows[o], b] += prediction_o(b) for every sample b: ``tod`` a
        float64 CUDA tensor (C, B) with unit stride along B; theta, phi, psi
        (B,) float32 or float64."""
        O = self.dims[3]
        if len(rows) != O:
            raise ValueError(f"need {O} output rows")
        if not (isinstance(tod, torch.Tensor) and tod.is_cuda and tod.dtype == torch.float64 and tod.dim() == 2
                and tod.stride(1) == 1):
            raise ValueError("tod must be a float64 (C, B) CUDA tensor with unit stride along B")
        if max(rows) >= tod.shape[0] or min(rows) < 0:
            raise ValueError("output row out of range")
        th, ph, ps = self._angles(theta, phi, psi)
        B = th.numel()
        if tod.shape[1] != B:
            raise ValueError("tod must have one column per sample")
        chunk = _pad(min(int(chunk), max(B, 1)))
        ws = self.workspace(chunk)
        r = (ctypes.c_int32 * O)(*[int(v) for v in rows])
        sc = (ctypes.c_double * O)(*[float(v) for v in self.scale])
        sh = (ctypes.c_double * O)(*[float(v) for v in self.shift])
        dt = _native.F32 if th.dtype == torch.float32 else _native.F64
        _native.check(_native.lib().todgpu_tail_accumulate(
            ctypes.byref(self.desc), th.data_ptr(), ph.data_ptr(), ps.data_ptr(), dt, B, r, sc, sh, tod.data_ptr(),
            tod.stride(0), chunk, ws.data_ptr(), ws.numel(), stream_handle()))
        return tod

    # -- state ----------------------------------------------------------------
    def state(self):
        """Host copy of everything needed to rebuild the network."""
        return dict(dims=np.array(self.dims), sigma=np.array(self.sigma), seed=np.array(self.seed),
                    params=self.params.cpu().numpy(), shift=self.shift, scale=self.scale,
                    freq=self.freq.cpu().numpy(), step=np.array(self.step))

    @classmethod
    def from_state(cls, st, device=None):
        F, H, D, O = (int(v) for v in st["dims"])
        net = cls(F, H, D, O, sigma=tuple(st["sigma"]), seed=int(st["seed"]), device=device)
        net.freq.copy_(torch.from_numpy(np.asarray(st["freq"], np.float32)))
        net.params.copy_(torch.from_numpy(np.asarray(st["params"], np.float32)))
        net.shift = np.asarray(st["shift"], np.float64)
        net.scale = np.asarray(st["scale"], np.float64)
        net.step = int(st["step"])
        net.sync_bf16()
        return net
