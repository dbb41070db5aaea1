"""Test-harness autograd wrapper: x = A^{-1} b on the device path, with the hand-written
adjoint (hm_solve_transpose) as the backward.  Used only by the tests."""
import numpy as np
import torch


class HodlrSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, b, handle):
        x = handle.solve(b.detach().cpu().numpy())
        ctx.handle = handle
        return torch.from_numpy(np.ascontiguousarray(x)).to(b)

    @staticmethod
    def backward(ctx, g):
        lam = ctx.handle.solve_transpose(g.detach().cpu().numpy())
        return torch.from_numpy(np.ascontiguousarray(lam)).to(g), None
