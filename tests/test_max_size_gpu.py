"""The largest lattice the 32-bit population offsets allow: 16384 x 14000
(9 x 16384 x 14000 = 2.06e9 < 2^31 elements per buffer).  A density bump
near the top-right corner (outlet and top wall) evolves for 20 steps; its
neighbourhood must equal, bit for bit, the same bump in a 256 x 128 lattice,
because every node runs the same arithmetic and nothing else reaches that
corner in 20 steps.  At 16384 nodes per row the limit is 14563 rows
(9 x 16384 x 14563 < 2^31 <= 9 x 16384 x 14564): that lattice is accepted
and one row more is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")

P = dict(collision=ip.MRT, storage=ip.F32, bc_set=ip.BC_CHANNEL, les_model=ip.LES_SMAGORINSKY, tau0=0.6,
         cs=0.1, u_in=0.0, rho0=1.0)


def corner_run(nx, ny, steps=20):
    rho = np.ones((ny, nx))
    yy, xx = np.mgrid[ny - 40:ny, nx - 60:nx]
    rho[ny - 40:, nx - 60:] += 1e-3 * np.exp(-((xx - (nx - 30)) ** 2 + (yy - (ny - 20)) ** 2) / 20.0)
    g = ip.Lattice(nx, ny, **P)
    g.init_macros(rho, None, None)
    del rho
    g.step(steps, 1)
    r = g.download(ip.FIELD_RHO)[ny - 64:, nx - 100:].copy()
    g.close()
    return r


def test_max_offset_lattice_matches_small_lattice_at_the_far_corner():
    big = corner_run(16384, 14000)
    small = corner_run(256, 128)
    assert np.abs(small - 1.0).max() > 1e-5  # the bump is there
    np.testing.assert_array_equal(big, small)


def test_lattice_beyond_offset_limit_is_refused():
    assert 9 * 16384 * 14563 < 2 ** 31 <= 9 * 16384 * 14564
    with pytest.raises(ip.IppiError, match="too large"):
        ip.Lattice(16384, 14564, **P)
    ip.Lattice(16384, 14563, **P).close()
