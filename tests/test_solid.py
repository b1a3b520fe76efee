"""Solid nodes on the FP64 oracle (CPU): halfway bounce-back on every fluid
link into a solid, and the momentum-exchange force of Mesh::OutputCd
(mesh.cpp:1461-1488)."""
import numpy as np
import pytest

import pyoracle as po
from ippi_lbm import scenes


def oracle(nx, ny, coll=po.MRT, les=1):
    o = po.Oracle(nx, ny, collision=coll, bc_set=po.BC_CHANNEL, les_model=les, tau0=0.56, cs=0.1,
                  u_in=0.05, delta_kernel=1, mdf_iters=1)
    return o


def test_solid_mask_checks():
    o = oracle(40, 20)
    m = np.zeros((20, 40), np.uint8)
    m[2, 10] = 1  # two nodes from the wall
    with pytest.raises(ValueError):
        o.set_solid(m)
    m[:] = 0
    m[10, 37] = 1  # two nodes from the outlet
    with pytest.raises(ValueError):
        o.set_solid(m)
    r = po.Oracle(40, 20, bc_set=po.BC_REF)
    m[:] = 0
    m[10, 10] = 1
    with pytest.raises(ValueError):
        r.set_solid(m)


def test_styles_of_solid_and_link_nodes():
    nx, ny = 48, 24
    o = oracle(nx, ny)
    m = scenes.cylinder_solid(nx, ny, 15.0, 12.0, 6)
    o.set_solid(m)
    st = o.get(po.FLAGS).astype(np.uint8)
    assert np.array_equal(st == ord("s"), m.astype(bool))
    near = np.zeros_like(m, bool)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            near |= np.roll(np.roll(m, dy, 0), dx, 1).astype(bool)
    assert np.array_equal(st == ord("b"), near & ~m.astype(bool))
    o.set_solid(None)
    assert not np.any(o.get(po.FLAGS) == ord("s"))


def test_at_rest_no_force_and_no_flow_through_solid():
    nx, ny = 48, 24
    o = po.Oracle(nx, ny, collision=po.MRT, bc_set=po.BC_CHANNEL, les_model=0, tau0=0.6, u_in=0.0)
    o.set_solid(scenes.cylinder_solid(nx, ny, 20.0, 12.0, 8))
    o.init_macros(np.ones((ny, nx)), np.zeros((ny, nx)), np.zeros((ny, nx)))
    assert o.step(20, 1) == 0
    np.testing.assert_allclose(o.solid_force(), 0.0, atol=1e-15)
    np.testing.assert_allclose(o.get(po.RHO), 1.0, atol=1e-14)


@pytest.mark.parametrize("coll", [po.BGK, po.MRT, po.RR])
def test_symmetric_solid_drag_positive_lift_zero(coll):
    """A solid symmetric about the channel centreline in the symmetric
    parabolic inflow: drag along +x (Re 20, Cd about 3.3), lift zero to
    rounding."""
    nx, ny = 80, 32
    o = oracle(nx, ny, coll, les=0)
    o.set_solid(scenes.cylinder_solid(nx, ny, 20.0, (ny - 1) / 2, 8))
    rho, ux, uy = scenes.channel_init(nx, ny, 0.05, noise=0.0)
    o.init_macros(rho, ux, uy)
    assert o.step(600, 1) == 0
    f = []
    for t in range(601, 1601, 10):  # the start-up sound waves still ring: average
        assert o.step(10, t) == 0
        f.append(o.solid_force())
    f = np.array(f)
    fx = f[:, 0].mean()
    assert fx > 1e-3
    assert np.abs(f[:, 1]).max() < 1e-12 * fx
    # the solid's nodes read as fluid at rest
    m = scenes.cylinder_solid(nx, ny, 20.0, (ny - 1) / 2, 8).astype(bool)
    assert np.all(o.get(po.UX)[m] == 0) and np.all(o.get(po.RHO)[m] == 1)
