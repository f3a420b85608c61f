"""A thin torch.autograd binding over cup2d_adjoint_run, for tests: the
objective of nsteps steps from a saved state, as a function of the initial
velocity (u0, v0) and of the body's velocity ub = (u, v, omega), whose
backward returns the discrete adjoint's gradients.  Each call restores the
checkpoint first, so repeated evaluations start from the same state."""
import torch


class AdjointObjective(torch.autograd.Function):
    @staticmethod
    def forward(fctx, u0, v0, ub, ctx, blob, nsteps, kwargs):
        ctx.restore(blob)
        ctx.set("u", u0.detach().cpu().numpy())
        ctx.set("v", v0.detach().cpu().numpy())
        ctx.set_shape(0, {"u": float(ub[0]), "v": float(ub[1]), "omega": float(ub[2])})
        need = any(fctx.needs_input_grad[:3])
        J, gu, gv, gb, dts, _ = ctx.adjoint(nsteps, gradient=need, **kwargs)
        fctx.dts = dts
        if need:
            fctx.save_for_backward(torch.from_numpy(gu), torch.from_numpy(gv), torch.from_numpy(gb))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(fctx, gJ):
        gu, gv, gb = fctx.saved_tensors
        return gJ * gu, gJ * gv, gJ * gb, None, None, None, None


def objective(ctx, blob, nsteps, u0, v0, ub, **kwargs):
    """J(u0, v0, ub) with autograd through the adjoint (kwargs: those of
    Context.adjoint other than nsteps and gradient, e.g. box, dt, every,
    w_energy, w_force)."""
    return AdjointObjective.apply(u0, v0, ub, ctx, blob, nsteps, kwargs)
