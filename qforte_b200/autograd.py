"""The dUCC energy as a differentiable torch function.

``ucc_energy(params, ducc)`` returns E(t) = <ref|U(t)^dag H U(t)|ref> for each
row of ``params`` ([nparam] or [batch, nparam], float64).  The forward pass is
one sweep of the device evaluator that prepares psi = U(t)|ref>, forms
sigma = H psi and reduces <psi|sigma>; the backward pass is the adjoint
reverse sweep of UCCVQE.measure_gradient (uccvqeabc.py:122-251): it un-applies
each exponential from psi and sigma in turn and reads 2 Re <sigma|K_mu|psi>
between them, so nothing but the final psi and sigma is kept between the two
passes.  Both run on the current torch stream.
"""

import ctypes

import torch

from ._lib import check, lib

__all__ = ["UCCEnergyFunction", "ucc_energy"]


def _use_current_stream():
    check(lib().qfb_set_stream(ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
          "qfb_set_stream")


class UCCEnergyFunction(torch.autograd.Function):

    @staticmethod
    def forward(ctx, params, ducc):
        P = params.detach()
        vec = P.dim() == 1
        P2 = P.reshape(-1, ducc.nparam).to(device="cuda", dtype=torch.float64).contiguous()
        ev = ducc.evaluator(P2.shape[0])
        _use_current_stream()
        d_par, d_en, _ = ev.tensors()
        d_par.copy_(P2)
        ev.run(0)
        E = d_en.clone()
        ctx.ev, ctx.gen, ctx.P2, ctx.vec = ev, ev.generation, P2, vec
        ctx.out_device = params.device
        return (E[0] if vec else E).to(params.device)

    @staticmethod
    def backward(ctx, gE):
        ev = ctx.ev
        _use_current_stream()
        d_par, _, d_grad = ev.tensors()
        if ev.generation != ctx.gen:  # another run reused the evaluator's states
            d_par.copy_(ctx.P2)
            ev.run(0)
        ev.run(2)
        G = d_grad.clone()
        g = gE.to(device="cuda", dtype=torch.float64).reshape(-1, 1) * G
        g = g[0] if ctx.vec else g
        return g.to(ctx.out_device), None


def ucc_energy(params, ducc):
    """Differentiable dUCC energies of ``ducc`` (a qforte_b200.ucc.DUCC)."""
    return UCCEnergyFunction.apply(params, ducc)
