"""Mechanical power of two heaving hemispheres and its gradient
(paper/Power.jl:13-83, the two-body design study).

The reference computes, for spheres of radius r1 with centres (0, 0, 0) and
(r1 + dx1, 0, 0), heave radiation on sphere 1 (A11, A12, B11, B12, assumed
symmetric), the diffraction and Froude-Krylov heave forces on both, the 2x2
equation of motion H Xi = F with H = w^2 (M + A) - i w (B + diag(B11)) + C,
and J = sum(1/2 B11 |i w Xi|^2) / (2/3 pi r1^3).  Its hydrostatics come from
Capytaine (paper/HydrostaticsRule.jl:7-15) and M = C there (Power.jl:18-19);
Capytaine is absent, so both are restated as the heave stiffness of a
hemisphere rho g pi r1^2 (rho = 1000, g = 9.81), keeping M = C.  As in the
reference, the radiation pressure uses rho = 1000 (Power.jl:40) and the
diffraction pressure rho = 1023 (:63), the Froude-Krylov pressure the default
rho = 1000 (src/waves.jl:150-153).

`two_body_power(..., grad=True)` returns dJ/d(r1, dx1, omega): the small
2x2 algebra is differentiated with torch autograd on the host (exact), the
boundary-element part with one `mh_hydro_batch_vjp` call, whose mesh
cotangent is pulled back to the generator parameters on the device
(`mh_mesh_param_vjp`): the two hemispheres are generated there.
"""
from __future__ import annotations

import math

import numpy as np

from ._native import default_context
from .api import GFWu, Rankine, RankineReflected
from .bodies import FloatingBody, hydro_batch
from .gradients import hydro_batch_vjp
from .meshgen import generate_combined, generate_hemisphere, generated_param_grad

RHO = 1000.0
RHO_DIFFRACTION = 1023.0
G = 9.81


def _bodies(r1, dx1, resolution, ctx):
    """The two heaving bodies (their dofs) and their mesh, generated on the
    device (parameters radius0, cx0, cy0, cz0, radius1, cx1, cy1, cz1)."""
    m1 = generate_hemisphere(r1, (0.0, 0.0, 0.0), resolution, ctx)
    m2 = generate_hemisphere(r1, (r1 + dx1, 0.0, 0.0), resolution, ctx)
    both = FloatingBody.rigid(m1, ["Heave"], body_name="sphere") + \
        FloatingBody.rigid(m2, ["Heave"], body_name="sphere")
    return both, generate_combined([m1, m2], ctx)


def _objective(A11, A12, B11, B12, F1r, F1i, F2r, F2i, K1r, K1i, K2r, K2i, w, r1):
    """Power.jl:15-80 after the boundary-element outputs (torch scalars)."""
    import torch

    C = RHO * G * math.pi * r1 ** 2
    M = C  # Power.jl:18-19
    Am = torch.stack([torch.stack([A11, A12]), torch.stack([A12, A11])])
    Bm = torch.stack([torch.stack([B11, B12]), torch.stack([B12, B11])])
    eye = torch.eye(2, dtype=torch.float64)
    inertia = M * eye + Am
    pto = torch.stack([B11, B11])
    resistance = Bm + torch.diag(pto)
    H = (w ** 2 * inertia).to(torch.complex128) - 1j * w * resistance.to(torch.complex128) \
        + (C * eye).to(torch.complex128)
    scale = RHO_DIFFRACTION / RHO
    F = torch.stack([torch.complex(scale * F1r + K1r, scale * F1i + K1i),
                     torch.complex(scale * F2r + K2r, scale * F2i + K2i)])
    Xi = torch.linalg.solve(H, F)
    P = 0.5 * pto * torch.abs(1j * w * Xi) ** 2
    return torch.sum(P) / ((2.0 / 3.0) * math.pi * r1 ** 3)


def two_body_power(r1: float = 1.0, dx1: float = 4.0, omega: float = 1.03, *, resolution=(32, 64),
                   green_functions=None, direct: bool = True, precision: str = "mixed",
                   tol: float = 1e-10, grad: bool = False, ctx=None):
    """J (and with grad=True a dict of dJ/dr1, dJ/ddx1, dJ/domega)."""
    import torch

    gfs = green_functions or (Rankine(), RankineReflected(), GFWu())
    ctx = ctx or default_context()
    body, mesh = _bodies(r1, dx1, resolution, ctx)
    dofs = list(body.dofs.values())
    om = np.array([omega])
    kw = dict(green_functions=gfs, direct=direct, precision=precision, tol=tol, rho=RHO, g=G, ctx=ctx)
    A, B, Fd, Fk, _ = hydro_batch(mesh, om, dofs, [0.0], **kw)
    # outputs used by Power.jl: radiation of sphere 1 (A[:, 0]), forces on both
    leaves = [A[0, 0, 0], A[1, 0, 0], B[0, 0, 0], B[1, 0, 0],
              Fd[0, 0, 0].real, Fd[0, 0, 0].imag, Fd[1, 0, 0].real, Fd[1, 0, 0].imag,
              Fk[0, 0, 0].real, Fk[0, 0, 0].imag, Fk[1, 0, 0].real, Fk[1, 0, 0].imag, omega, r1]
    t = [torch.tensor(float(v), dtype=torch.float64, requires_grad=grad) for v in leaves]
    J = _objective(*t)
    if not grad:
        return float(J)
    J.backward()
    g = [float(x.grad) for x in t]
    bA = np.zeros_like(A)
    bB = np.zeros_like(B)
    bF = np.zeros_like(Fd)
    bK = np.zeros_like(Fk)
    bA[0, 0, 0], bA[1, 0, 0], bB[0, 0, 0], bB[1, 0, 0] = g[0], g[1], g[2], g[3]
    bF[0, 0, 0] = g[4] + 1j * g[5]
    bF[1, 0, 0] = g[6] + 1j * g[7]
    bK[0, 0, 0] = g[8] + 1j * g[9]
    bK[1, 0, 0] = g[10] + 1j * g[11]
    r = hydro_batch_vjp(mesh, om, dofs, [0.0], bA, bB, bF, bK, **kw)
    p = generated_param_grad(mesh, r.mesh)
    # r1 scales both bodies and moves the second centre (x = r1 + dx1)
    grads = {"r1": g[13] + p["radius0"] + p["radius1"] + p["cx1"], "dx1": p["cx1"],
             "omega": g[12] + float(r.omegas[0])}
    return float(J.detach()), grads


def optimize_two_body_power(r0: float = 2.0, dx0: float = 3.0, lower=(1.0, 1.0), upper=(4.0, 4.0), *,
                            omega: float = 1.03, iterations: int = 100, g_tol: float = 1e-3, callback=None,
                            **kw) -> dict:
    """Maximise the two-body power over (r1, dx1) in a box
    (paper/optimization.jl: J = power(r, dx), start (2, 3), bounds [1, 4]^2,
    100 iterations, gradient tolerance 1e-3).  Each evaluation is one
    ``two_body_power(..., grad=True)``: the forward batch and its adjoint on
    the device.  The reference runs Optim's Fminbox(LBFGS()) (a barrier for
    the box around L-BFGS); this uses scipy's L-BFGS-B, whose box handling is
    a projection, so the two take different paths to the same bounded
    optimum.  ``kw`` goes to ``two_body_power`` (resolution, precision,
    green functions, ctx).  ``callback(x, J)`` sees every accepted iterate.
    Returns {"x": (r1, dx1), "power", "iterations", "evaluations",
    "history": [(r1, dx1, power) per iterate], "converged", "message"}."""
    from scipy.optimize import minimize

    history = []
    evals = [0]
    cache = {}

    def f(x):
        key = (float(x[0]), float(x[1]))
        if key not in cache:
            J, g = two_body_power(key[0], key[1], omega, grad=True, **kw)
            evals[0] += 1
            cache[key] = (-J, np.array([-g["r1"], -g["dx1"]]))
        return cache[key]

    def on_iterate(xk):
        J = -f(xk)[0]
        history.append((float(xk[0]), float(xk[1]), J))
        if callback is not None:
            callback(np.array(xk, dtype=np.float64), J)

    x0 = np.array([r0, dx0], dtype=np.float64)
    history.append((r0, dx0, -f(x0)[0]))
    res = minimize(f, x0, jac=True, method="L-BFGS-B", bounds=list(zip(lower, upper)),
                   callback=on_iterate, options=dict(maxiter=int(iterations), gtol=float(g_tol)))
    return {"x": (float(res.x[0]), float(res.x[1])), "power": float(-res.fun), "iterations": int(res.nit),
            "evaluations": evals[0], "history": history, "converged": bool(res.success),
            "message": str(res.message)}
