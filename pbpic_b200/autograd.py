"""PyTorch autograd wrapper of the differentiable form (pbpic_diff_* in the C ABI).

HarrisLoss.apply(params, engine) returns the engine's loss of a GEM Harris sheet
run -- the time-integrated magnetic energy, or the time-integrated work j.E the
electric field does on the particles -- as a function of params = (psi0, nb,
Ti/Te), a float64 tensor of 3 values; its backward pass runs the library's
discrete adjoint (checkpointed, recomputed between checkpoints) and returns
d loss / d params.
"""
import ctypes

import torch

from . import _lib as L


class DiffEngine:
    """One checkpointed forward/adjoint engine on the current CUDA device."""

    def __init__(self, mx, my, ppc, nsteps, checkpoint_every, precision="fp32", dx=0.1, mime=25.0, wpe_wce=2.0,
                 lam=0.5, nb0=0.2, cfl=0.5, seed=3, loss="magnetic"):
        self._lib = L.lib()
        prec = {"fp64": L.FP64_PLAIN, "fp32": L.FP32_MIXED}[precision]
        kind = {"magnetic": L.LOSS_MAGNETIC, "jdote": L.LOSS_JDOTE}[loss]
        self.cfg = L.DiffConfig(mx=mx, my=my, ppc=ppc, precision=prec, dx=dx, mime=mime, wpe_wce=wpe_wce,
                                lambda_=lam, nb0=nb0, cfl=cfl, nsteps=nsteps, checkpoint_every=checkpoint_every,
                                loss=kind, seed=seed)
        self._h = ctypes.c_void_p()
        L.check(self._lib.pbpic_diff_create(ctypes.byref(self.cfg), ctypes.byref(self._h)))

    def forward(self, psi0, nb, ti_te):
        loss = ctypes.c_double()
        prm = L.DiffParams(psi0=float(psi0), nb=float(nb), ti_te=float(ti_te))
        L.check(self._lib.pbpic_diff_forward(self._h, ctypes.byref(prm), ctypes.byref(loss)))
        return loss.value

    def backward(self):
        g = (ctypes.c_double * 3)()
        L.check(self._lib.pbpic_diff_backward(self._h, g))
        return [g[0], g[1], g[2]]

    def close(self):
        if self._h:
            self._lib.pbpic_diff_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class HarrisLoss(torch.autograd.Function):
    """loss(psi0, nb, Ti/Te) with the adjoint as its backward pass."""

    @staticmethod
    def forward(ctx, params, engine):
        p = params.detach().to("cpu", torch.float64)
        loss = engine.forward(p[0].item(), p[1].item(), p[2].item())
        ctx.engine = engine
        return torch.tensor(loss, dtype=torch.float64, device=params.device)

    @staticmethod
    def backward(ctx, grad_out):
        g = torch.tensor(ctx.engine.backward(), dtype=torch.float64, device=grad_out.device)
        return grad_out * g, None
