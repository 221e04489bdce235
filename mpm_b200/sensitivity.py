"""Gradients of simulation outcomes with respect to material parameters.

Two routes through the FP64 USL step, giving the same derivative:

* forward mode (``Solver.set_sensitivities``): each step carries, with every
  particle, node and cell-slot quantity, its derivatives with respect to up to
  two material parameters; the terminal Jacobian d x_final / d theta is at
  hand when the run ends (``TerminalPositions``);
* reverse mode (``Solver.adjoint_record`` / ``adjoint_reverse``): the run
  keeps checkpoints, and one reverse sweep of the step's adjoint gives, for
  one loss, its gradient with respect to the parameters and to the whole
  initial state (positions, velocities, stresses) (``AdjointPositions``).
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


def adjoint_gradient(build, theta, params, nsteps, x_target, checkpoint_every=0):
    """(loss, dL/dtheta) of L = sum |x_final - x_target|^2 by the reverse sweep."""
    s = build(theta)
    loss, g = s.adjoint_run(nsteps, params, x_target, checkpoint_every)
    s.close()
    return loss, g


if torch is not None:
    class AdjointPositions(torch.autograd.Function):
        """x_final = f(theta); backward runs the adjoint's reverse sweep with the
        incoming gradient as dL/dx_final.

        forward(theta, build, params, nsteps, checkpoint_every): records the
        run (checkpoints every ``checkpoint_every`` steps) and returns the final
        particle positions (float64 tensor, n x dim)."""

        @staticmethod
        def forward(ctx, theta, build, params, nsteps, checkpoint_every=0):
            s = build(theta.detach().cpu().numpy())
            s.adjoint_record(nsteps, params, checkpoint_every)
            ctx.solver = s
            return torch.from_numpy(np.ascontiguousarray(s.read()["x"]))

        @staticmethod
        def backward(ctx, grad_x):
            r = ctx.solver.adjoint_reverse(dL_dx=grad_x.detach().cpu().numpy())
            ctx.solver.close()
            return torch.from_numpy(r["params"]), None, None, None, None
