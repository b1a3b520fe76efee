"""The alternative LES closures of Mesh::CaculateLESTau (WALE, coherent
structure, wall-damped Cs; mesh.cpp:934-1071, 2113-2146) on the FP64 oracle:
closed-form values on states whose velocity gradient is known."""
import numpy as np
import pytest

import pyoracle as po

NX, NY, TAU0 = 48, 24, 0.56


def oracle(les):
    return po.Oracle(NX, NY, collision=po.MRT, bc_set=po.BC_CHANNEL, les_model=les, tau0=TAU0, cs=0.1,
                     u_in=0.05, delta_kernel=1)


def interior(a):
    # nodes whose forward differences are all taken (x < nx - 1, y < ny - 2)
    return a[: NY - 2, : NX - 1]


def test_wale_vanishes_in_pure_shear():
    o = oracle(4)
    yy, xx = np.mgrid[0:NY, 0:NX].astype(float)
    o.init_macros(np.ones((NY, NX)), 1e-3 * yy, np.zeros((NY, NX)))
    np.testing.assert_allclose(interior(o.get(po.TAU)), TAU0, rtol=0, atol=1e-15)


def test_wale_of_pure_strain():
    a = 1e-3
    o = oracle(4)
    yy, xx = np.mgrid[0:NY, 0:NX].astype(float)
    o.init_macros(np.ones((NY, NX)), a * xx, -a * yy)
    ss = 2 * a * a                     # S:S
    gg = 2 * (a * a / 3) ** 2          # Gd:Gd, Gd = diag(a^2/3, a^2/3)
    want = TAU0 + 3 * 0.45 ** 2 * gg ** 1.5 / (ss ** 2.5 + gg ** 1.25 + 1e-12)
    np.testing.assert_allclose(interior(o.get(po.TAU)), want, rtol=1e-12)
    # in the last column the x differences are 0: g = diag(0, -a)
    ss, gg = a * a, 5 * a ** 4 / 9
    want = TAU0 + 3 * 0.45 ** 2 * gg ** 1.5 / (ss ** 2.5 + gg ** 1.25 + 1e-12)
    np.testing.assert_allclose(o.get(po.TAU)[: NY - 2, NX - 1], want, rtol=1e-12)


def test_closures_on_equilibrium_state_give_tau0():
    """At equilibrium Pi_neq = 0: the coherent and wall-damped closures add
    nothing (their eddy viscosity scales with Pi_neq)."""
    yy, xx = np.mgrid[0:NY, 0:NX].astype(float)
    for les in (5, 6):
        o = oracle(les)
        if les == 6:
            o.set_wall_distance(np.full((NY, NX), 10.0))
        o.init_macros(np.ones((NY, NX)), 1e-3 * xx, -1e-3 * yy)
        np.testing.assert_allclose(o.get(po.TAU), TAU0, atol=1e-15)


def test_wall_damping_and_missing_distance():
    o = oracle(6)
    assert o.step(1, 1) == -1  # no wall distance yet
    rng = np.random.default_rng(0)
    rho, ux, uy = 1 + rng.normal(0, 1e-3, (NY, NX)), rng.normal(0, 1e-2, (NY, NX)), rng.normal(0, 1e-2, (NY, NX))
    taus = []
    for d in (-5.0, 3.0, 30.0):
        o = oracle(6)
        o.set_wall_distance(np.full((NY, NX), d))
        o.init_macros(rho, ux, uy)
        assert o.step(2, 1) == 0
        taus.append(o.get(po.TAU))
    # Cs = 3 / (1 + 1.71828^(6 - d)) grows with the distance; tau with it
    assert np.all(taus[0] <= taus[1]) and np.all(taus[1] <= taus[2])
    assert np.all(taus[0] - TAU0 < 1e-3 * (taus[2] - TAU0).max())
    assert (taus[2] - TAU0).max() > 1e-3
