"""Seeded uneven design batch (splitmix64 population) and its radius
derivatives through the forward mode."""
from __future__ import annotations

import numpy as np
import pytest


def test_splitmix64_known_values(mh):
    # splitmix64 from seed 0: the published first outputs of the generator
    g = mh.SplitMix64(0)
    assert [g.next_u64() for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_population_shape(mh):
    pop = mh.designs(seed=0, count=48)
    assert len(pop) == 48
    assert all(0.5 <= d.radius <= 2.0 for d in pop)
    assert all(8 <= d.resolution[0] <= 40 and d.resolution[1] == 2 * d.resolution[0] for d in pop)
    nf = [((d.resolution[0] + 1) // 2) * d.resolution[1] for d in pop]
    assert min(nf) >= 64 and max(nf) <= 1640
    assert mh.designs(seed=0, count=48)[5] == pop[5]  # reproducible


@pytest.mark.gpu
def test_design_batch_radius_derivatives(mh, gpu):
    pop = [mh.Design(0.7, (8, 16)), mh.Design(1.6, (10, 20))]
    om = np.linspace(0.3, 3.0, 6)
    res = mh.design_batch(pop, om, precision="mixed", tol=1e-13, ctx=gpu)
    h = 1e-6
    for d, r in zip(pop, res):
        p = mh.design_batch([mh.Design(d.radius + h, d.resolution)], om, precision="fp64", ctx=gpu)[0]
        m = mh.design_batch([mh.Design(d.radius - h, d.resolution)], om, precision="fp64", ctx=gpu)[0]
        for got, a, b in ((r.d_added_mass_dR, p.added_mass, m.added_mass), (r.d_damping_dR, p.damping, m.damping)):
            fd = (a - b) / (2 * h)
            assert np.max(np.abs(got - fd)) <= 1e-6 * np.max(np.abs(fd))


@pytest.mark.gpu
def test_design_batch_concurrent_contexts_match_serial(mh, gpu):
    """Four worker threads with a context each give, design by design, the
    serial results (bit for bit: every call is deterministic).  Meshes of 64
    to 1640 panels in flight together also exercise kernels whose dynamic
    shared memory depends on the size (one process-wide limit per kernel)."""
    pop = mh.designs(seed=3, count=24, ntheta=(8, 40))
    om = np.linspace(0.3, 3.0, 8)
    serial = mh.design_batch(pop, om, precision="mixed", tol=1e-12, ctx=gpu)
    conc = mh.design_batch(pop, om, precision="mixed", tol=1e-12, workers=4)
    ctxs = [mh.Context(0) for _ in range(3)]
    try:
        given = mh.design_batch(pop, om, precision="mixed", tol=1e-12, contexts=ctxs)
    finally:
        for c in ctxs:
            c.close()
    for a, b, c in zip(serial, conc, given):
        assert a.design == b.design == c.design and a.nfaces == b.nfaces == c.nfaces
        for f in ("added_mass", "damping", "d_added_mass_dR", "d_damping_dR"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
            assert np.array_equal(getattr(a, f), getattr(c, f)), f
