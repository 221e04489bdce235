"""Gradients of simulation outcomes with respect to material parameters.

The library differentiates the FP64 USL step in forward mode: each step
carries, with every particle, node and cell-slot quantity, its derivatives
with respect to up to two material parameters (``Solver.set_sensitivities``).
For a handful of parameters this gives the exact gradient of any function of
the final state at about three times the cost of the run, with no checkpoints
and no reverse sweep: the terminal Jacobian d x_final / d theta is at hand
when the run ends, and the backward pass of ``TerminalPositions`` contracts it
with the incoming gradient.
"""
import numpy as np

try:
    import torch
except ImportError:  # torch is optional for the library itself
    torch = None


def run_with_sensitivities(build, theta, params, nsteps):
    """Build a solver for parameter values ``theta`` (``build(theta)`` returns
    a set-up, initialised Solver), run ``nsteps`` carrying derivatives with
    respect to ``params`` ([(material_id, kind), ...]), and return
    (x_final (n, dim), J (n_params, n, dim))."""
    s = build(theta)
    s.set_sensitivities(params)
    s.step(nsteps)
    x = s.read()["x"]
    J = s.read_sensitivities("x")[:len(params)]
    s.close()
    return x, J


if torch is not None:
    class TerminalPositions(torch.autograd.Function):
        """x_final = f(theta) with d x_final / d theta from the tangent run.

        forward(theta, build, params, nsteps): theta a 1-D tensor of parameter
        values in the units of ``params``' kinds; returns the final particle
        positions (float64 tensor, n x dim).  backward contracts the incoming
        gradient with the stored terminal Jacobian."""

        @staticmethod
        def forward(ctx, theta, build, params, nsteps):
            x, J = run_with_sensitivities(build, theta.detach().cpu().numpy(), params, nsteps)
            ctx.save_for_backward(torch.from_numpy(J))
            return torch.from_numpy(x)

        @staticmethod
        def backward(ctx, grad_x):
            (J,) = ctx.saved_tensors
            g = (J * grad_x.to(J.dtype).unsqueeze(0)).sum(dim=(1, 2))
            return g, None, None, None
