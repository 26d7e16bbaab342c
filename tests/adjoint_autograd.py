"""torch.autograd.Function around the discrete adjoint (test harness only).

J(U0) = kinetic energy of the state after `nsteps` ENO-Roe steps from U0;
the backward pass is the C ABI's reverse sweep (frozen ENO choices and dt)."""
import torch


class KineticEnergyAfterSteps(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, adj, nsteps, dt0):
        adj.upload(U0.detach().cpu().double().numpy())
        J = adj.forward(nsteps, dt0)
        ctx.adj = adj
        return torch.tensor(J, dtype=torch.float64, device=U0.device)

    @staticmethod
    def backward(ctx, gJ):
        ctx.adj.backward()
        g = torch.from_numpy(ctx.adj.gradient()).to(gJ.device)
        return gJ * g, None, None, None


def kinetic_energy_after_steps(U0, adj, nsteps, dt0):
    return KineticEnergyAfterSteps.apply(U0, adj, nsteps, dt0)
