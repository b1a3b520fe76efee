"""The IB forcing term of each collision operator (oracle, FP64): one forced
collision with the equilibrium at u* + F/(2 rho) must add exactly F to the
node's momentum and nothing to its mass, and the viscous-stress part of the
source must carry the (1 - 1/(2 tau)) factor."""
import ctypes as C

import numpy as np
import pytest

import pyoracle as po

EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1.0])
EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1.0])
WK = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def feq(rho, ux, uy):
    e = EX * ux + EY * uy
    return WK * rho * (1 + 3 * e + 4.5 * e * e - 1.5 * (ux * ux + uy * uy))


def ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@pytest.mark.parametrize("coll", [po.BGK, po.MRT, po.RR])
def test_forced_collision_adds_the_force_to_the_momentum(oracle, coll):
    L = oracle.lib()
    rng = np.random.default_rng(coll)
    for _ in range(50):
        rho = 1 + rng.uniform(-1e-2, 1e-2)
        u = rng.uniform(-0.05, 0.05, 2)
        f = feq(rho, *u) + rng.normal(0, 1e-3, 9)
        rho = f.sum()
        us = np.array([(f * EX).sum(), (f * EY).sum()]) / rho
        F = rng.uniform(-1e-3, 1e-3, 2)
        tau0 = 0.52
        tau = tau0 if coll == po.BGK else rng.uniform(0.51, 0.8)
        ue = us + F / (2 * rho)
        out = np.zeros(9)
        L.orc_collide_node(coll, ptr(f), rho, ue[0], ue[1], tau, ptr(out))
        lf = np.zeros(9)
        L.orc_force_node(coll, ue[0], ue[1], F[0], F[1], tau0, tau, ptr(lf))
        post = out + lf
        assert post.sum() == pytest.approx(rho, abs=1e-14)
        mom = np.array([(post * EX).sum(), (post * EY).sum()])
        np.testing.assert_allclose(mom - rho * us, F, rtol=0, atol=1e-15)
        # mass- and momentum-free source; its stress part is (1 - 1/(2 tau)) (uF + Fu)
        assert abs(lf.sum()) < 1e-16
        if coll != po.BGK:
            pxy = (lf * EX * EY).sum()
            assert pxy == pytest.approx((1 - 0.5 / tau) * (ue[0] * F[1] + ue[1] * F[0]), rel=1e-9,
                                        abs=1e-18)
