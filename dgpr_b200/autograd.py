"""torch.autograd wrappers over the adjoint entry points of the C ABI.

`integrate(U0, solver, scheme, dt, nsteps, slots)` advances a device state
(torch float64 CUDA tensor in the reference layout U[e][r][b]) by nsteps RK
steps through dgb_forward_record; its backward is dgb_backward_device, the
hand-written discrete adjoint with binomial checkpointing.  With
`theta` = [mu, source[0..4]] or [mu, source[0..4], Tw] (a float64 tensor of
6 or 7; Tw: the isothermal walls' temperature) the run uses those parameters
(dgb_set_params, dgb_set_wall_temperature) and is differentiable in them too
(dgb_backward_params_device).  `residual(U,
solver)` is f = -Minv R(U) with dgb_residual_vjp_device as its backward.

Both run the native library only; there is no torch compute path.  A solver
handle holds one recorded run at a time: calling `integrate` again on the same
solver before the first result's backward makes that backward raise.
"""
import torch

from . import DgbError, ERR_ARG

__all__ = ["integrate", "residual", "STAGES"]

# `slots` value for integrate(): keep every state and every RK stage state,
# so the backward sweep recomputes nothing (dgb_forward_record_stages)
STAGES = -1


def _dev_f64(t, n, what):
    if not (t.is_cuda and t.dtype == torch.float64):
        raise TypeError(f"{what} must be a float64 CUDA tensor")
    if t.numel() != n:
        raise ValueError(f"{what} has {t.numel()} values, the solver's state has {n}")
    return t.contiguous()


class _Integrate(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, solver, scheme, dt, nsteps, slots):
        U0 = _dev_f64(U0, solver.n, "U0")
        torch.cuda.current_stream().synchronize()
        solver.set_state_device(U0.data_ptr())
        if slots == STAGES:
            solver.forward_record_stages(scheme, dt, nsteps, norms=False)
        else:
            solver.forward_record(scheme, dt, nsteps, slots, norms=False)
        UN = torch.empty_like(U0)
        solver.get_state_device(UN.data_ptr())
        ctx.solver = solver
        ctx.record_id = solver.record_id
        return UN

    @staticmethod
    def backward(ctx, gUN):
        solver = ctx.solver
        if getattr(solver, "record_id", None) != ctx.record_id:
            raise DgbError(ERR_ARG, "the solver recorded another run since this one; its adjoint is gone")
        gUN = _dev_f64(gUN, solver.n, "grad")
        torch.cuda.current_stream().synchronize()
        g0 = torch.empty_like(gUN)
        solver.backward_device(gUN.data_ptr(), g0.data_ptr())
        return g0, None, None, None, None, None


class _IntegrateParams(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, theta, solver, scheme, dt, nsteps, slots):
        from . import Params
        th = [float(v) for v in theta.detach().cpu().reshape(-1)]
        if len(th) not in (6, 7):
            raise ValueError("theta must hold [mu, source[0..4]] or [mu, source[0..4], Tw]")
        p = Params.from_array(solver.params.as_array())
        p.mu = th[0]
        for r in range(5):
            p.source[r] = th[1 + r]
        solver.set_params(p)
        if len(th) == 7:
            solver.set_wall_temperature(th[6])
        UN = _Integrate.forward(ctx, U0, solver, scheme, dt, nsteps, slots)
        ctx.theta_like = theta
        return UN

    @staticmethod
    def backward(ctx, gUN):
        solver = ctx.solver
        if getattr(solver, "record_id", None) != ctx.record_id:
            raise DgbError(ERR_ARG, "the solver recorded another run since this one; its adjoint is gone")
        gUN = _dev_f64(gUN, solver.n, "grad")
        torch.cuda.current_stream().synchronize()
        g0 = torch.empty_like(gUN)
        dpar = torch.empty(7, dtype=torch.float64, device=gUN.device)
        solver.backward_params_device(gUN.data_ptr(), g0.data_ptr(), dpar.data_ptr())
        solver.synchronize()
        k = ctx.theta_like.numel()
        gth = dpar[:k].to(device=ctx.theta_like.device, dtype=ctx.theta_like.dtype).reshape(ctx.theta_like.shape)
        return g0, gth, None, None, None, None, None


class _Residual(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, solver):
        U = _dev_f64(U, solver.n, "U")
        torch.cuda.current_stream().synchronize()
        f = torch.empty_like(U)
        solver.residual_device(U.data_ptr(), 0, f.data_ptr())
        solver.synchronize()
        ctx.solver = solver
        ctx.save_for_backward(U)
        return f

    @staticmethod
    def backward(ctx, g):
        (U,) = ctx.saved_tensors
        solver = ctx.solver
        g = _dev_f64(g, solver.n, "grad")
        torch.cuda.current_stream().synchronize()
        out = torch.empty_like(U)
        solver.residual_vjp_device(U.data_ptr(), g.data_ptr(), out.data_ptr())
        solver.synchronize()
        return out, None


def integrate(U0, solver, scheme, dt, nsteps, slots=None, theta=None):
    """U_N after nsteps RK steps from U0, differentiable in U0.  slots: number
    of state checkpoints held on the device (default: every state), or STAGES
    to keep every stage state as well.  theta: optional float64 tensor
    [mu, source[0..4]] or [mu, source[0..4], Tw] of the run's parameters,
    then also differentiable."""
    slots = int(slots if slots is not None else nsteps)
    if theta is None:
        return _Integrate.apply(U0, solver, int(scheme), float(dt), int(nsteps), slots)
    return _IntegrateParams.apply(U0, theta, solver, int(scheme), float(dt), int(nsteps), slots)


def residual(U, solver):
    """f = -Minv R(U), differentiable in U."""
    return _Residual.apply(U, solver)
