"""The Poisson negative log-likelihood of ROI images and its adjoint gradient (iscu_nll_*), behind a
torch.autograd.Function for checking: forward runs the likelihood kernel, backward the adjoint kernel, which recomputes
each emitter's field instead of storing per-emitter PSFs.

Parameters: per emitter (x, y) in ROI pixels, z defocus in nm, N photons; one background per frame; the Zernike
coefficients (waves rms, Noll indices of the spec). The model is documented in include/iscu.h (iscu_nll_spec).

Across ranks (one process per GPU) the frames split into contiguous ranges (shard_problem): the emitters and
backgrounds of a frame live on one rank, so their gradients stay local, and the one exchange is the sum of the NLL
and of the Zernike gradient over the ranks (reduce_shared: one all-reduce of 1 + J float64 values).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._abi import NllSpec as _NllSpecC
from .engine import Engine, IscuError, _ptr, _require_tensor, check


@dataclass
class NllSpec:
    wavelength_nm: float = 670.0
    na: float = 1.45
    n_imm: float = 1.518
    pixel_nm: float = 108.0
    roi: int = 32
    os: int = 2
    pupil: int = 32
    noll: tuple = tuple(range(4, 25))

    def c(self) -> _NllSpecC:
        s = _NllSpecC()
        s.wavelength_nm, s.na, s.n_imm, s.pixel_nm = self.wavelength_nm, self.na, self.n_imm, self.pixel_nm
        s.roi, s.os, s.pupil, s.n_zern = self.roi, self.os, self.pupil, len(self.noll)
        for i, j in enumerate(self.noll):
            s.noll[i] = j
        return s


class NllModel:
    """iscu_nll_model on an engine's device."""

    def __init__(self, engine: Engine, spec: NllSpec):
        self.engine = engine
        self.lib = engine.lib
        self.spec = spec
        h = C.c_void_p()
        cs = spec.c()
        check(self.lib.iscu_nll_model_create(engine.h, C.byref(cs), C.byref(h)))
        self.h = h
        kappa, nz = C.c_double(), C.c_int32()
        check(self.lib.iscu_nll_model_info(h, C.byref(kappa), C.byref(nz)))
        self.kappa, self.n_zern = kappa.value, nz.value
        engine._plans.add(self)

    def close(self):
        if self.h:
            if self.engine.h:
                self.lib.iscu_nll_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_dev(self, params, frame, bg, zern, counts, nll, err, g_params=None, g_bg=None, g_zern=None, mu=None,
                sync=True):
        """iscu_nll_eval_dev on prepared CUDA tensors (params (n, 4) float32, frame int32, bg float32, counts float32,
        nll 1 float64, err 1 int32; the gradient outputs when g_params is given); zern a float64 numpy array. Every
        buffer is checked (dtype, device, contiguity, size) before the call, so none is read or written past."""
        import torch
        n, nf, R, dev = int(params.shape[0]), int(bg.shape[0]), self.spec.roi, self.engine.device
        if not (isinstance(zern, np.ndarray) and zern.dtype == np.float64 and zern.flags.c_contiguous
                and zern.size == self.n_zern):
            raise ValueError(f"zern must be a C-contiguous float64 array of {self.n_zern} coefficients")
        _require_tensor(params, "params", (torch.float32,), dev, 4 * n)
        _require_tensor(frame, "frame", (torch.int32,), dev, n)
        _require_tensor(bg, "bg", (torch.float32,), dev, nf)
        _require_tensor(counts, "counts", (torch.float32,), dev, n * R * R)
        _require_tensor(nll, "nll", (torch.float64,), dev, 1)
        _require_tensor(err, "err", (torch.int32,), dev, 1)
        if mu is not None:
            _require_tensor(mu, "mu", (torch.float32,), dev, n * R * R)
        if g_params is not None:
            _require_tensor(g_params, "g_params", (torch.float32,), dev, 4 * n)
            _require_tensor(g_bg, "g_bg", (torch.float64,), dev, nf)
            _require_tensor(g_zern, "g_zern", (torch.float64,), dev, self.n_zern)
        self.engine._before(sync)
        check(self.lib.iscu_nll_eval_dev(self.h, params.shape[0], _ptr(params), _ptr(frame), bg.shape[0], _ptr(bg),
                                         zern.ctypes.data_as(C.POINTER(C.c_double)), _ptr(counts), _ptr(mu),
                                         _ptr(nll), _ptr(g_params), _ptr(g_bg), _ptr(g_zern), _ptr(err)))
        self.engine._after(sync)

    def evaluate(self, params, frame, bg, zern, counts, grad=False, want_mu=False):
        """params (n, 4) float32, frame (n,) int32, bg (F,) float32, counts (n, R, R) float32: CUDA tensors; zern
        (J,) float64 (any). Returns (nll float, mu | None, (g_params (n, 4) float32, g_bg (F,) float64, g_zern (J,)
        float64) | None)."""
        import torch
        dev = params.device
        params = params.detach().to(torch.float32).contiguous()
        frame = frame.to(torch.int32).contiguous()
        bg = bg.detach().to(torch.float32).contiguous()
        counts = counts.to(torch.float32).contiguous()
        z = np.ascontiguousarray(np.asarray(zern.detach().cpu() if hasattr(zern, "detach") else zern,
                                            dtype=np.float64))
        n, nf, R = params.shape[0], bg.shape[0], self.spec.roi
        if params.numel() != 4 * n or frame.numel() != n or counts.numel() != n * R * R or z.size != self.n_zern:
            raise ValueError(f"expected params (n, 4), frame (n,), counts (n, {R}, {R}) and {self.n_zern} Zernike "
                             f"coefficients; got {tuple(params.shape)}, {tuple(frame.shape)}, {tuple(counts.shape)}, "
                             f"{z.size}")
        nll = torch.zeros(1, dtype=torch.float64, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        mu = torch.empty_like(counts) if want_mu else None
        g = (torch.empty_like(params), torch.empty(nf, dtype=torch.float64, device=dev),
             torch.empty(len(z), dtype=torch.float64, device=dev)) if grad else (None, None, None)
        self.engine._before(True)
        check(self.lib.iscu_nll_eval_dev(self.h, n, _ptr(params), _ptr(frame), nf, _ptr(bg),
                                         z.ctypes.data_as(C.POINTER(C.c_double)), _ptr(counts), _ptr(mu), _ptr(nll),
                                         _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), _ptr(err)))
        self.engine._after(True)
        if int(err.item()):
            raise IscuError(1, "an emitter names a frame outside the batch")   # ISCU_ERR_ARG
        return float(nll.item()), mu, (g if grad else None)


def poisson_nll(model: NllModel, params, bg, zern, counts, frame):
    """The NLL as a differentiable torch scalar (float64) in params (n, 4), bg (F,) and zern (J,)."""
    import torch

    class _PoissonNll(torch.autograd.Function):
        @staticmethod
        def forward(ctx, params, bg, zern):
            value, _, _ = model.evaluate(params, frame, bg, zern, counts)
            ctx.save_for_backward(params, bg, zern)
            return torch.tensor(value, dtype=torch.float64, device=params.device)

        @staticmethod
        def backward(ctx, gout):
            params, bg, zern = ctx.saved_tensors
            _, _, (gp, gb, gz) = model.evaluate(params, frame, bg, zern, counts, grad=True)
            go = gout.to(torch.float64)
            return ((go * gp.to(torch.float64)).to(params.dtype), (go * gb).to(bg.dtype),
                    (go.to(zern.device) * gz.to(zern.device)).to(zern.dtype))

    return _PoissonNll.apply(params, bg, zern)


def shard_problem(prob, rank: int, world: int):
    """The rank's share of an NllProblem: its contiguous range of frames (insiliscope_b200.shard.frame_range), their
    emitters and backgrounds, frames renumbered from 0; `frame0` (the range's first frame) keys the rank's noise draws
    as the whole problem's. The Zernike coefficients are shared by every rank."""
    from dataclasses import replace

    from .shard import frame_range
    F = len(prob.bg)
    first, end = frame_range(rank, world, F)
    sel = (prob.frame >= first) & (prob.frame < end)
    return replace(prob, frame=(prob.frame[sel] - first).astype(np.int32), params_true=prob.params_true[sel],
                   bg_true=prob.bg_true[first:end], params=prob.params[sel], bg=prob.bg[first:end],
                   frame0=prob.frame0 + first)


def reduce_shared(packed):
    """Sums, in place over the ranks, a float64 tensor holding [NLL, d/dzern (J)] (the only gradient every rank
    contributes to); returns it. One all-reduce; a no-op without an initialised process group of 2 or more ranks."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(packed, op=dist.ReduceOp.SUM)
    return packed
