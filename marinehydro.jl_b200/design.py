"""Uneven design batch: many hemispheres of different radii and panel
counts, each with its added mass, damping and their derivatives with
respect to the radius over a set of frequencies.

This is the sensitivity study of the reference's paper scripts
(paper/CoeficientsGradients.jl, paper/MeshGradients_singlebody.jl, which
differentiate A and B of a hemisphere with respect to its radius), run over
a seeded population of designs.  The derivatives come from one forward-mode
call per mesh (``hydro_batch_jvp`` along the exact radius tangent of the
generated mesh): every frequency's dA/dR and dB/dR at the cost of one extra
tangent solve on the forward factors.

Designs are drawn with splitmix64 (Steele, Lea, Flood 2014: state += 0x9e37
79b97f4a7c15; z = (z ^ z>>30) * 0xbf58476d1ce4e5b9; z = (z ^ z>>27) *
0x94d049bb133111eb; z ^ z>>31), U(0,1) = (z >> 11) * 2^-53:
radius ~ U(0.5, 2.0), n_theta ~ U{8..40}, n_phi = 2 n_theta.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .api import ExactGuevelDelhommeau, Rankine, RankineReflected
from .bodies import FloatingBody
from ._native import default_context
from .gradients import hydro_batch_jvp
from .meshgen import generate_hemisphere, generated_tangent

_MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & _MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))


@dataclass
class Design:
    radius: float
    resolution: tuple


def designs(seed: int = 0, count: int = 48, radius=(0.5, 2.0), ntheta=(8, 40)) -> list:
    """The seeded population: radius ~ U(radius), n_theta ~ U{ntheta}, n_phi = 2 n_theta."""
    g = SplitMix64(seed)
    out = []
    for _ in range(count):
        r = radius[0] + (radius[1] - radius[0]) * g.uniform()
        nt = ntheta[0] + min(int(g.uniform() * (ntheta[1] - ntheta[0] + 1)), ntheta[1] - ntheta[0])
        out.append(Design(r, (nt, 2 * nt)))
    return out


@dataclass
class DesignResult:
    design: Design
    nfaces: int
    added_mass: np.ndarray  # (n_omega,) heave
    damping: np.ndarray
    d_added_mass_dR: np.ndarray
    d_damping_dR: np.ndarray


def _one_design(d: Design, om, gfs, precision, tol, ctx) -> DesignResult:
    # the mesh and its radius tangent made on the device (no host generation
    # or upload on the design loop's host threads)
    mesh = generate_hemisphere(d.radius, (0.0, 0.0, 0.0), d.resolution, ctx=ctx or default_context())
    body = FloatingBody.rigid(mesh, ["Heave"])
    tan = generated_tangent(mesh, "radius")
    r = hydro_batch_jvp(mesh, om, list(body.dofs.values()), (), tan, green_functions=gfs,
                        precision=precision, tol=tol, ctx=ctx)
    return DesignResult(d, mesh.nfaces, r.added_mass[0, 0].copy(), r.damping[0, 0].copy(),
                        r.d_added_mass[0, 0].copy(), r.d_damping[0, 0].copy())


def design_batch(population, omegas, *, green_functions=None, precision="mixed", tol=1e-10, ctx=None,
                 workers: int = 1, device: int = 0, contexts=None) -> list:
    """Heave A, B and dA/dR, dB/dR of every design at every frequency, in
    the population's order.

    ``workers > 1`` runs that many host threads, each with its own library
    context (its own CUDA streams and workspace) on ``device``, taking the
    designs largest first from a shared queue: small meshes leave most of the
    GPU idle one at a time, and distinct contexts run concurrently (the
    library calls release the GIL).  Every design's result is the same as
    in a serial run (each call is deterministic and independent).
    ``contexts`` (a list of ``Context``) gives the workers instead: one
    thread per context, reused across calls, so their workspaces and
    Delhommeau tables are built once rather than per call."""
    gfs = green_functions or (Rankine(), RankineReflected(), ExactGuevelDelhommeau())
    om = np.asarray(omegas, dtype=np.float64)
    pop = list(population)
    if contexts is not None:
        contexts = list(contexts)
        workers = len(contexts)
    if workers <= 1 or len(pop) <= 1:
        c = contexts[0] if contexts else ctx
        return [_one_design(d, om, gfs, precision, tol, c) for d in pop]
    import threading

    from ._native import Context

    # largest first (panels ~ n_theta^2), so the last designs taken are short
    order = sorted(range(len(pop)), key=lambda q: -pop[q].resolution[0] * pop[q].resolution[1])
    res = [None] * len(pop)
    errors = []
    lock = threading.Lock()
    nxt = [0]

    def run(given):
        c = given if given is not None else Context(device)
        try:
            while True:
                with lock:
                    if nxt[0] >= len(order) or errors:
                        return
                    q = order[nxt[0]]
                    nxt[0] += 1
                res[q] = _one_design(pop[q], om, gfs, precision, tol, c)
        except BaseException as e:  # noqa: BLE001 - re-raised in the caller's thread
            with lock:
                errors.append(e)
        finally:
            if given is None:
                c.close()

    nt = min(int(workers), len(pop))
    threads = [threading.Thread(target=run, args=(contexts[t] if contexts else None,)) for t in range(nt)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    if errors:
        raise errors[0]
    return res
