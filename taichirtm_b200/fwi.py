"""Differentiable P-SV modelling: seismograms as a torch function of (vp, vs,
rho) with gradients from the exact discrete adjoint (librtm_b200
``rtm_forward_checkpointed`` + ``rtm_adjoint``).

The reference has no gradient; this is the FWI extension of its forward
operator (src/forward_modeling.py:309-453): the forward is the reference's
step exactly, and the adjoint differentiates that discrete step (sponge,
interior masks, point sources and receivers included), so finite
differences of the same discrete forward are the check.

Memory: the forward stores the full wavefield every ``ckpt_every`` steps
(default round(sqrt(nt))); the backward recomputes one segment at a time."""
import ctypes
import math

import numpy as np
import torch

from . import _lib
from .fields import to_tensor
from .plan import PSV, Plan, ShotGeometry, _i32p, _ptr, _stream, check


class FWIProblem:
    """Fixed acquisition for gradient evaluations: grid, shots (windows and
    LOCAL source/receiver indices), wavelets (3, nsrc_total, nt)."""

    def __init__(self, nx, nz, dx, dz, fs, nt, absorbing_frame, shots, wavelets, ckpt_every=None,
                 surface=None, tune=None, device=None, ckpt_dtype="f32"):
        """tune: launch shape dict, None (library default) or "auto" (timed on
        short gradients of this acquisition, cached per GPU and geometry)."""
        self.device = torch.device(device if device is not None else "cuda")
        self.nx, self.nz, self.nt = int(nx), int(nz), int(nt)
        if tune == "auto":  # time candidate launch shapes on short gradients (cached)
            from . import autotune

            def make(t, steps):
                w = to_tensor(wavelets, torch.float32, self.device)[..., :steps].contiguous()
                return FWIProblem(nx, nz, dx, dz, fs, steps, absorbing_frame, shots, w,
                                  ckpt_every=max(1, round(math.sqrt(steps))), surface=surface, tune=t,
                                  device=self.device, ckpt_dtype=ckpt_dtype)
            tune = autotune.best_fwi_shape(make, self.nx, self.nz, list(shots)) if self.nt >= autotune.FWI_TUNE_STEPS else None
        self.tune = tune
        self.plan = Plan(nx, nz, dx, dz, nt, fs, absorbing_frame, PSV, list(shots), tune=tune,
                         device=self.device)
        self.wavelets = to_tensor(wavelets, torch.float32, self.device)
        self.ckpt_every = int(ckpt_every or max(1, round(math.sqrt(nt))))
        self.ckpt_dtype = _lib.CKPT_DTYPES[ckpt_dtype]
        self.surface = None if surface is None else to_tensor(surface, torch.float32, self.device)
        L = _lib.lib()
        self.n_ckpt = int(L.rtm_plan_num_checkpoints(self.plan.h, self.ckpt_every))
        self.state_floats = int(L.rtm_plan_state_floats(self.plan.h))

    def checkpoint_bytes(self):
        return int(_lib.lib().rtm_plan_checkpoint_bytes(self.plan.h, self.ckpt_every, self.ckpt_dtype))

    def forward(self, lam, mu, rho):
        """Set the model, run the checkpointed forward.  Returns (seis (3,
        nrec_total, nt), checkpoint buffer, flags)."""
        self.plan.set_model(mu, lam, rho, self.surface)
        ck = torch.empty(max(self.checkpoint_bytes(), 1), dtype=torch.uint8, device=self.device)
        seis = torch.empty((3, self.plan.nrec_total, self.nt), dtype=torch.float32, device=self.device)
        flags = np.zeros(len(self.plan.shots), np.int32)
        with torch.cuda.device(self.device):
            check(_lib.lib().rtm_forward_checkpointed(self.plan.h, _ptr(self.wavelets), _ptr(seis),
                                                      self.ckpt_every, self.ckpt_dtype, _ptr(ck), 100,
                                                      _i32p(flags), _stream()), "rtm_forward_checkpointed")
        return seis, ck, flags

    def adjoint(self, resid, ck, want_wavelet_grad=False):
        """Gradients (5, nx, nz) float64 w.r.t. (lam, mu, mxz, inv_rho_u,
        inv_rho_w) and optionally dJ/d(wavelets) (3, nsrc_total, nt)."""
        r = to_tensor(resid, torch.float32, self.device)
        grad = torch.zeros((5, self.nx, self.nz), dtype=torch.float64, device=self.device)
        gw = (torch.zeros_like(self.wavelets) if want_wavelet_grad and self.plan.nsrc_total else None)
        with torch.cuda.device(self.device):
            check(_lib.lib().rtm_adjoint(self.plan.h, _ptr(self.wavelets), _ptr(r), self.ckpt_every,
                                         self.ckpt_dtype, _ptr(ck), _ptr(grad), _ptr(gw), _stream()),
                  "rtm_adjoint")
        return grad, gw

    def close(self):
        self.plan.close()


def chain_to_lame_rho(grad, mu, rho):
    """Map gradients w.r.t. the derived coefficients to (lam, mu, rho).

    mxz(i,j) = 4 / sum of 1/mu over (i,j),(i+1,j),(i,j+1),(i+1,j+1)  (fm:271-276)
      d mxz / d mu_k = mxz^2 / (4 mu_k^2)
    inv_rho_u(i,j) = 2 / (rho(i,j) + rho(i+1,j)),  inv_rho_w with (i,j+1)  (fm:288-307)
      d inv_rho_u / d rho = -inv_rho_u^2 / 2 for both cells.
    Interior cells only, as the coefficients are interior-only."""
    g_lam = grad[0].clone()
    g_mu = grad[1].clone()
    g_rho = torch.zeros_like(g_mu)
    mu = mu.to(torch.float64)
    rho = rho.to(torch.float64)
    a, b, c, d = mu[1:-1, 1:-1], mu[2:, 1:-1], mu[1:-1, 2:], mu[2:, 2:]
    mxz = 4.0 / (1.0 / a + 1.0 / b + 1.0 / c + 1.0 / d)
    w = grad[2][1:-1, 1:-1] * mxz * mxz / 4.0
    g_mu[1:-1, 1:-1] += w / (a * a)
    g_mu[2:, 1:-1] += w / (b * b)
    g_mu[1:-1, 2:] += w / (c * c)
    g_mu[2:, 2:] += w / (d * d)
    bu = 2.0 / (rho[1:-1, 1:-1] + rho[2:, 1:-1])
    bw = 2.0 / (rho[1:-1, 1:-1] + rho[1:-1, 2:])
    tu = -0.5 * grad[3][1:-1, 1:-1] * bu * bu
    tw = -0.5 * grad[4][1:-1, 1:-1] * bw * bw
    g_rho[1:-1, 1:-1] += tu + tw
    g_rho[2:, 1:-1] += tu
    g_rho[1:-1, 2:] += tw
    return g_lam, g_mu, g_rho


class _Seismograms(torch.autograd.Function):
    @staticmethod
    def forward(ctx, lam, mu, rho, problem):
        seis, ck, flags = problem.forward(lam.detach(), mu.detach(), rho.detach())
        if int(flags.max()) != 0:
            raise FloatingPointError(f"forward propagation became non-finite (codes {flags.tolist()})")
        ctx.problem = problem
        ctx.ck = ck
        ctx.save_for_backward(mu.detach(), rho.detach())
        return seis

    @staticmethod
    def backward(ctx, g_seis):
        mu, rho = ctx.saved_tensors
        grad, _ = ctx.problem.adjoint(g_seis.contiguous(), ctx.ck)
        ctx.ck = None
        g_lam, g_mu, g_rho = chain_to_lame_rho(grad, mu, rho)
        return g_lam.to(mu.dtype), g_mu.to(mu.dtype), g_rho.to(rho.dtype), None


def seismograms(vp, vs, rho, problem: FWIProblem):
    """(3, nrec_total, nt) seismograms, differentiable w.r.t. vp, vs, rho
    (material as the reference builds it, src/rtm.py:901-902:
    mu = rho vs^2, lam = rho vp^2 - 2 mu)."""
    mu = rho * vs * vs
    lam = rho * vp * vp - 2.0 * mu
    return _Seismograms.apply(lam, mu, rho, problem)


def l2_misfit(vp, vs, rho, problem: FWIProblem, observed, components=(0, 2)):
    """0.5 ||d - d_obs||^2 on the given components (0 = vx/u, 2 = vz/w)."""
    d = seismograms(vp, vs, rho, problem)
    obs = to_tensor(observed, torch.float32, d.device)
    r = d[list(components)] - obs[list(components)]
    return 0.5 * (r.double() ** 2).sum()
