"""Gradient of the sinogram Poisson log-likelihood (mcpet_grad) and a
torch.autograd binding of it.

    L(A, s) = sum_b y_b ln(lambda_b) - lambda_b,
    lambda  = trues + scatter (the transport of activity A through the
              phantom with voxel densities s_v * rho_v) + background.

dL/dA comes from event back-tallying, dL/ds from the path-replay score
function (see include/mcpet.h, mcpet_grad).  Tensors live on the scene's
CUDA device; the computation is the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _abi
from ._abi import check, lib
from .scene import RunOptions, Scene


@dataclass
class GradResult:
    loglik: float
    grad_activity: Optional["object"]       # torch tensor [n_voxels] or None
    grad_density_scale: Optional["object"]  # torch tensor [n_voxels] or None
    tallies: dict                           # forward run: trues, scatter, ... (torch, device)
    events: int
    replayed: int
    mismatches: int
    forward_ms: float
    gradient_ms: float


def _device_tallies(scene: Scene, torch, dev) -> dict:
    cfg, info = scene.config, scene.info
    return {
        "trues": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "scatter": torch.zeros(int(cfg.n_bins), dtype=torch.int32, device=dev),
        "image_trues": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "image_scatter": torch.zeros(int(info.n_voxels), dtype=torch.int32, device=dev),
        "spectrum": torch.zeros(max(cfg.n_energy_bins, 1), dtype=torch.int32, device=dev),
        "psf_count": torch.zeros(1, dtype=torch.int32, device=dev),
        "histories": torch.zeros(1, dtype=torch.int64, device=dev),
        "coincidences": torch.zeros(1, dtype=torch.int64, device=dev),
    }


def grad(scene: Scene, measured, background=None, opts: Optional[RunOptions] = None, activity: bool = True,
         density: bool = True, event_buffer=None, tallies: Optional[dict] = None) -> GradResult:
    """Forward transport + log-likelihood + gradient.  measured/background:
    float32 CUDA tensors of n_bins; event_buffer: optional uint8 CUDA tensor
    (24 bytes per tallied coincidence) whose records stay readable after."""
    import torch
    opts = opts or RunOptions()
    dev = measured.device
    nv = int(scene.info.n_voxels)
    t = tallies if tallies is not None else _device_tallies(scene, torch, dev)
    ga = torch.zeros(nv, dtype=torch.float32, device=dev) if activity else None
    gs = torch.zeros(nv, dtype=torch.float32, device=dev) if density else None
    d = _abi.Tallies()
    d.trues, d.scatter = t["trues"].data_ptr(), t["scatter"].data_ptr()
    d.image_trues, d.image_scatter = t["image_trues"].data_ptr(), t["image_scatter"].data_ptr()
    d.spectrum = t["spectrum"].data_ptr()
    d.psf_count = t["psf_count"].data_ptr()
    d.total_histories = t["histories"].data_ptr()
    d.coincidences = t["coincidences"].data_ptr()
    a = _abi.GradArgs()
    a.measured = measured.contiguous().data_ptr()
    a.background = None if background is None else background.contiguous().data_ptr()
    a.grad_activity = None if ga is None else ga.data_ptr()
    a.grad_density_scale = None if gs is None else gs.data_ptr()
    if event_buffer is not None:
        a.event_buffer = event_buffer.data_ptr()
        a.event_capacity = event_buffer.numel() // _abi.EVENT_RECORD_BYTES
    co = opts.to_c()
    check(lib().mcpet_grad(scene.handle, C.byref(co), C.byref(d), C.byref(a)))
    return GradResult(a.loglik, ga, gs, t, int(a.events), int(a.replayed), int(a.mismatches), a.forward_ms,
                      a.gradient_ms)


def event_records(buf, n: int) -> np.ndarray:
    """Decode the first n records of an event buffer (uint8 tensor) into a
    structured array: rng_x, rng_y, voxel, bin."""
    dt = np.dtype([("rng_x", "<i4"), ("rng_y", "<i4"), ("voxel", "<u4"), ("pad", "<u4"), ("bin", "<i8")])
    raw = buf[: n * _abi.EVENT_RECORD_BYTES].cpu().numpy()
    return raw.view(dt)


def _autograd_function():
    import torch

    class PoissonLogLikelihood(torch.autograd.Function):
        """L(activity, density_scale) for a scene; backward gives dL/dA and
        dL/ds.  The forward sets the scene's activity from `activity` and is
        evaluated at the scene's own densities, i.e. density_scale must be
        all ones (the derivative is taken there)."""

        @staticmethod
        def forward(ctx, activity, density_scale, scene, measured, background, opts):
            if not bool(torch.all(density_scale == 1)):
                raise ValueError("density_scale must be 1 (the forward runs at the scene's densities)")
            scene.set_activity(activity.detach().float().cpu().numpy())
            r = grad(scene, measured, background, opts)
            ctx.save_for_backward(r.grad_activity, r.grad_density_scale)
            ctx.devices = (activity.device, density_scale.device)
            ctx.stats = r
            return torch.tensor(r.loglik, dtype=torch.float64, device=measured.device)

        @staticmethod
        def backward(ctx, g):
            ga, gs = ctx.saved_tensors
            gf = g.to(torch.float32)
            da, ds = ctx.devices
            return (ga * gf).to(da), (gs * gf).to(ds), None, None, None, None

    return PoissonLogLikelihood


def poisson_loglik(activity, density_scale, scene: Scene, measured, background=None,
                   opts: Optional[RunOptions] = None):
    """torch.autograd entry: L as a 0-d float64 tensor differentiable in
    activity and density_scale."""
    return _autograd_function().apply(activity, density_scale, scene, measured, background, opts)
