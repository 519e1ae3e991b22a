"""Design gradients of a WaveBot buoy (src/meshes.jl:458-479): the adjoint's
mesh cotangents dotted with the exact WaveBot tangents give dJ/d(r1, r2, d1,
d2); checked against central differences of regenerated meshes and against
the forward mode along the same tangent."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = dict(r1=0.88, r2=0.35, d1=0.16, d2=0.37)
KW = dict(n_points=(3, 4, 3), n_theta=12)


def _gfs(mh):
    return (mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())


def _weights(nd, nw, nb, seed=5):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=(nd, nd, nw)), rng.normal(size=(nd, nd, nw)),
            rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb)))


def _J(mh, gpu, mesh, om, dofs, betas, w):
    A, B, Fd, _, _ = mh.hydro_batch(mesh, om, dofs, betas, green_functions=_gfs(mh), precision="fp64", ctx=gpu)
    wA, wB, wF = w
    return float(np.sum(wA * A) + np.sum(wB * B) + np.real(np.sum(np.conj(wF) * Fd)))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_wavebot_design_gradients(mh, gpu, precision):
    mesh = mh.wavebot_mesh(**P, **KW)
    # translational modes: constant motion fields, the same on every mesh
    dofs = [mh.translational_dofs(mesh, "Heave"), mh.translational_dofs(mesh, "Surge")]
    om = np.array([0.8, 1.6])
    betas = [0.0]
    w = _weights(2, len(om), 1)
    r = mh.hydro_batch_vjp(mesh, om, dofs, betas, w[0], w[1], w[2], None, green_functions=_gfs(mh),
                           precision=precision, tol=1e-13, ctx=gpu)
    tan = mh.wavebot_tangents(**P, **KW)
    h = 1e-6
    for name in ("r1", "r2", "d1", "d2"):
        g = r.mesh.dot(tan[name])
        jp = _J(mh, gpu, mh.wavebot_mesh(**{**P, name: P[name] + h}, **KW), om, dofs, betas, w)
        jm = _J(mh, gpu, mh.wavebot_mesh(**{**P, name: P[name] - h}, **KW), om, dofs, betas, w)
        fd = (jp - jm) / (2 * h)
        assert abs(g - fd) <= 1e-5 * max(abs(fd), abs(g)), (name, g, fd)
        # forward mode along the same mesh tangent
        t = mh.hydro_batch_jvp(mesh, om, dofs, betas, t_mesh=tan[name], green_functions=_gfs(mh),
                               precision=precision, tol=1e-13, ctx=gpu)
        jt = float(np.sum(w[0] * t.d_added_mass) + np.sum(w[1] * t.d_damping)
                   + np.real(np.sum(np.conj(w[2]) * t.d_diffraction)))
        assert abs(jt - g) <= 1e-8 * max(abs(g), 1e-300), (name, jt, g)
