"""torch.autograd.Function over the C-ABI: per-case overload loss of the power flow
as a function of the bus injections, with the backward pass by mpf_adjoint.

    L = PowerFlowLoss.apply(p, q, pf, cases, precision)   # p, q: (n_cases, n_bus) float64
    L.sum().backward()                                    # p.grad, q.grad from J^T lambda

The grid, its outages and the ratings (pf.set_ratings) are fixed; p and q replace the
net injections of every bus in every case.  Cases that do not converge give L = 0 and
zero gradients (check pf.results().status).
"""
import numpy as np
import torch

from . import _types as T


class PowerFlowLoss(torch.autograd.Function):
    @staticmethod
    def forward(ctx, p, q, pf, cases, precision=T.MIXED):
        sbus = torch.stack([p.detach(), q.detach()], -1).cpu().numpy()
        pf.set_cases(cases, sbus=sbus)
        pf.solve(T.NR, precision)
        res = pf.results()
        over = pf.branch_flows()["overload"]
        over = np.where(res.status == T.CASE_CONVERGED, over, 0.0)
        ctx.pf = pf
        ctx.precision = precision
        return torch.as_tensor(over, dtype=torch.float64, device=p.device)

    @staticmethod
    def backward(ctx, grad_out):
        g = ctx.pf.adjoint(ctx.precision)
        w = grad_out.detach().cpu().numpy()[:, None]
        gp = torch.as_tensor(g["grad_p"] * w, device=grad_out.device)
        gq = torch.as_tensor(g["grad_q"] * w, device=grad_out.device)
        return gp, gq, None, None, None
