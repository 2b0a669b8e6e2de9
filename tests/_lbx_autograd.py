"""torch.autograd.Function over the C-ABI adjoint pair (test harness only):
forward = lbx_adjoint_forward, backward = lbx_adjoint_backward."""
import numpy as np
import torch

import lbx


class PlaneObjective(torch.autograd.Function):
    """J(gx, tau, tau_s, profile_b) for a fixed lattice, mask, run length and
    objective; the inputs are FP64 tensors (scalars and an LX*LY profile)."""

    @staticmethod
    def forward(ctx, gx, tau, tau_s, profile, setup):
        p = setup["params"]
        lp = lbx.Params(**{**p, "gaccel": (float(gx), 0.0, 0.0, 0.0, 0.0, 0.0),
                           "tau": (float(tau), float(tau_s))})
        dom = lbx.Domain(lp, setup["mask"])
        dom.set_face_profile(False, profile.detach().cpu().numpy())
        dom.init_equilibrium(0, 1.0, 0.0, 0.0, 0.0)
        dom.init_equilibrium(1, 0.0, 0.0, 0.0, 0.0)
        J = dom.adjoint_forward(0, setup["steps"], setup["K"], setup["plane"],
                                setup["t_first"], setup["steps"], setup["w_c"], setup["w_ux"])
        ctx.dom = dom
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        g = ctx.dom.adjoint_backward(profile_b=True)
        ctx.dom.close()
        s = float(gJ)
        return (torch.tensor(s * g["d_gaccel"][0], dtype=torch.float64),
                torch.tensor(s * g["d_tau"], dtype=torch.float64),
                torch.tensor(s * g["d_tau_s"], dtype=torch.float64),
                torch.from_numpy(s * g["d_profile_b"]), None)
