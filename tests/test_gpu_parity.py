"""Parity of the sm_100a step kernels (through the C ABI) with the FP64 oracle.

FP64 storage runs the reference's arithmetic in double: populations and
moments must agree with the oracle to 1e-12 relative to the field's scale;
FP32 to 1e-5 after one step from the same state (the tolerance the method
states for FP32) and to 1e-4 after tens of steps.  Node flags must match
bit for bit.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402

NETS = {t: np.fromfile(os.path.join(GOLDEN, "band_nets", f"AutoT0{t}.f32"), dtype=np.float32)
        for t in (1, 3, 5, 7)}


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pair(nx, ny, storage=ip.F64, **kw):
    coll = kw.get("collision", 0)
    bc = kw.get("bc_set", 0)
    ok = dict(collision=coll, bc_set=bc, les_model=kw.get("les_model", 1),
              tau0=kw.get("tau0", 0.55), cs=kw.get("cs", 0.173), u_in=kw.get("u_in", 0.1),
              rho0=1.0, plate_x0=kw.get("plate_x0", 400), avg_start=kw.get("avg_start", 30000),
              delta_kernel=kw.get("delta_kernel", 1), mdf_iters=kw.get("mdf_iters", 1))
    o = po.Oracle(nx, ny, **ok)
    g = ip.Lattice(nx, ny, storage=storage, **ok)
    return o, g


FIELDS = [(po.F, ip.FIELD_F), (po.RHO, ip.FIELD_RHO), (po.UX, ip.FIELD_UX), (po.UY, ip.FIELD_UY),
          (po.TAU, ip.FIELD_TAU)]


def compare(o, g, tol, fields=FIELDS):
    """Max difference over the lattice, relative to each field's scale:
    populations to max|f|, density to 1, velocities to max|u_x| (the flow's
    velocity scale; u_y alone can be pure round-off), tau absolute."""
    worst = {}
    uscale = max(float(np.abs(o.get(po.UX)).max()), 1e-12)
    for fo, fg in fields:
        a, b = g.download(fg), o.get(fo)
        d = float(np.abs(a - b).max())
        scale = {ip.FIELD_F: float(np.abs(b).max()), ip.FIELD_RHO: 1.0, ip.FIELD_UX: uscale,
                 ip.FIELD_UY: uscale, ip.FIELD_TAU: 1.0}[fg]
        worst[fg] = d / scale
        assert worst[fg] <= tol, (fg, worst[fg])
    return worst


@pytest.mark.parametrize("coll", [ip.BGK, ip.MRT, ip.RR])
def test_plate_fp64_matches_oracle(coll):
    o, g = pair(416, 12, collision=coll, tau0=0.53, avg_start=10)
    assert np.array_equal(g.download(ip.FIELD_FLAGS), o.get(po.FLAGS).astype(np.uint8))
    compare(o, g, 1e-12)  # initial state
    for n in (1, 9, 15):
        assert o.step(n, 1) == 0
        g.step(n, 1)
        compare(o, g, 1e-12)
    for fo, fg in [(po.AVG_U, ip.FIELD_AVG_U), (po.AVG_V, ip.FIELD_AVG_V),
                   (po.AVG_RHO, ip.FIELD_AVG_RHO)]:
        assert rel(g.download(fg), o.get(fo)) < 1e-12


def test_plate_fp64_with_boundary_nets():
    o, g = pair(416, 12, tau0=0.52)
    for t, w in NETS.items():
        o.load_band_net(t, w)
        g.load_band_net(t, w)
    for n in (1, 4, 10):
        o.step(n, 1)
        g.step(n, 1)
        # the nets run in FP32 (as libtorch does); summation order differs
        compare(o, g, 2e-6)
        assert np.array_equal(g.download(ip.FIELD_NNFLAG), o.get(po.NNFLAG))


def test_boundary_net_outputs_match_torch_forward():
    """The nets' outputs themselves (tau where a net set it, after one step
    from rest and after a few): the tensor-core evaluation (FP16 hi/lo
    operand parts, FP32 sums) against the oracle's FP32 forward, pinned to
    torch's outputs, within 5e-7 absolute on outputs near 0.5 (8 FP32 ulp;
    1.2e-7 measured on a B200)."""
    o, g = pair(416, 12, tau0=0.52)
    for t, w in NETS.items():
        o.load_band_net(t, w)
        g.load_band_net(t, w)
    worst = 0.0
    for n in (1, 3):
        o.step(n, 1)
        g.step(n, 1)
        flag = g.download(ip.FIELD_NNFLAG)
        assert np.array_equal(flag, o.get(po.NNFLAG))
        net = flag > 0
        assert net.any()
        worst = max(worst, float(np.abs(g.download(ip.FIELD_TAU)[net] - o.get(po.TAU)[net]).max()))
    print(f"largest net-output difference {worst:.3e}")
    assert worst <= 5e-7


def test_plate_fp32_one_step_tolerance():
    o, g = pair(416, 24, storage=ip.F32, collision=ip.MRT, tau0=0.53)
    rng = np.random.default_rng(1)
    ux = 0.05 + rng.uniform(-1e-2, 1e-2, (24, 416))
    uy = rng.uniform(-1e-2, 1e-2, (24, 416))
    rho = 1 + rng.uniform(-1e-3, 1e-3, (24, 416))
    o.init_macros(rho, ux, uy)
    g.init_macros(rho, ux, uy)
    o.step(1, 1)
    g.step(1, 1)
    compare(o, g, 1e-5)
    o.step(30, 2)
    g.step(30, 2)
    compare(o, g, 1e-4)


def cylinder_markers(cx, cy, r, n):
    th = 2 * np.pi * np.arange(n) / n
    return np.stack([cx + r * np.sin(th), cy + r * np.cos(th)], axis=1)


@pytest.mark.parametrize("coll,kern", [(ip.BGK, ip.DELTA_PESKIN4), (ip.MRT, ip.DELTA_PESKIN4),
                                       (ip.RR, ip.DELTA_BILINEAR)])
def test_channel_cylinder_fp64_matches_oracle(coll, kern):
    nx, ny = 160, 48
    o, g = pair(nx, ny, collision=coll, bc_set=ip.BC_CHANNEL, u_in=0.05, tau0=0.56,
                cs=0.1, delta_kernel=kern, mdf_iters=2)
    xy = cylinder_markers(40.3, 24.1, 6.0, 38)
    ds = np.full(38, 2 * np.pi * 6 / 38)
    o.set_markers(xy, ds=ds)
    g.set_markers(xy, ds=ds)
    y = np.arange(ny) + 0.5
    ux = np.tile((4 * 0.05 * y * (ny - y) / ny ** 2)[:, None], (1, nx))
    rng = np.random.default_rng(0)
    ux = ux + rng.uniform(-1e-4, 1e-4, ux.shape)
    o.init_macros(np.ones((ny, nx)), ux, np.zeros((ny, nx)))
    g.init_macros(np.ones((ny, nx)), ux, np.zeros((ny, nx)))
    for n in (1, 20, 40):
        o.step(n, 1)
        g.step(n, 1)
        compare(o, g, 1e-11)
        fo, mo = o.forces()
        fg, mg = g.forces(with_mass=True)
        np.testing.assert_allclose(fg, fo, rtol=1e-10, atol=1e-14)
        assert abs(mg - mo) / mo < 1e-13


def test_channel_fp32_cylinder_forces():
    nx, ny = 160, 48
    o, g = pair(nx, ny, storage=ip.F32, collision=ip.MRT, bc_set=ip.BC_CHANNEL, u_in=0.05,
                tau0=0.56, cs=0.1, delta_kernel=ip.DELTA_PESKIN4)
    xy = cylinder_markers(40.3, 24.1, 6.0, 38)
    o.set_markers(xy)
    g.set_markers(xy)
    o.step(200, 1)
    g.step(200, 1)
    compare(o, g, 2e-4)
    np.testing.assert_allclose(g.forces(), o.forces()[0], rtol=2e-3)


@pytest.mark.parametrize("storage", [ip.F16, ip.BF16])
def test_half_storage_runs_and_conserves_mass(storage):
    nx, ny = 256, 64
    g = ip.Lattice(nx, ny, storage=storage, collision=ip.MRT, bc_set=ip.BC_CHANNEL, u_in=0.04,
                   tau0=0.55, cs=0.1)
    r = ip.Lattice(nx, ny, storage=ip.F64, collision=ip.MRT, bc_set=ip.BC_CHANNEL, u_in=0.04,
                   tau0=0.55, cs=0.1)
    g.step(400, 1)
    r.step(400, 1)
    u, ur = g.download(ip.FIELD_UX), r.download(ip.FIELD_UX)
    tol = 2e-3 if storage == ip.F16 else 3e-2
    assert rel(u, ur) < tol
    _, m = g.forces(with_mass=True)
    _, mr = r.forces(with_mass=True)
    assert abs(m - mr) / mr < (1e-4 if storage == ip.F16 else 2e-3)


def test_graph_and_single_launches_agree():
    a = ip.Lattice(300, 40, storage=ip.F32, collision=ip.RR, tau0=0.6)
    b = ip.Lattice(300, 40, storage=ip.F32, collision=ip.RR, tau0=0.6)
    a.step(6, 1)
    for t in range(1, 7):
        b.step(1, t)
    assert np.array_equal(a.download(ip.FIELD_F), b.download(ip.FIELD_F))


@pytest.mark.parametrize("storage", [ip.F32, ip.F64])
def test_net_step_chain_matches_side_stream_form(storage):
    """The plate step with boundary nets runs prep, nets and bulk kernels as
    a chain of programmatic dependent launches; the timed form
    (ippi_profile_steps) runs the same kernels with the nets on a side
    stream joined by events.  Both orders must give the same bits: the nets
    read prep's moments only after its grid completed, and the step ends
    only after the nets."""
    (_, a), (_, b) = pair(416, 24, storage, tau0=0.52), pair(416, 24, storage, tau0=0.52)
    for t, w in NETS.items():
        a.load_band_net(t, w)
        b.load_band_net(t, w)
    a.step(12, 1)
    b.profile_steps(12, 1)
    for fld in (ip.FIELD_F, ip.FIELD_TAU, ip.FIELD_NNFLAG):
        assert np.array_equal(a.download(fld), b.download(fld))


def test_divergence_is_reported_not_faulted():
    g = ip.Lattice(64, 16, storage=ip.F64)
    rho = np.ones((16, 64))
    rho[8, 30] = 20.0
    g.init_macros(rho)
    with pytest.raises(ip.DivergedError):
        g.step(3, 1)


def test_bad_arguments_are_rejected():
    with pytest.raises(ip.IppiError):
        ip.Lattice(64, 16, tau0=0.5)
    g = ip.Lattice(64, 32, bc_set=ip.BC_CHANNEL, u_in=0.05, tau0=0.6)
    with pytest.raises(ip.IppiError):
        g.set_markers(cylinder_markers(3.0, 16.0, 2.0, 8))  # stencil leaves the interior
    with pytest.raises(ip.IppiError):
        g.load_band_net(1, np.zeros(10, np.float32))
    rho = np.ones((32, 64))
    rho[5, 7] = 0.0
    with pytest.raises(ip.IppiError, match=r"node 327\b"):
        g.init_macros(rho)
    ux = np.zeros((32, 64))
    ux[31, 63] = np.nan
    with pytest.raises(ip.IppiError, match=r"node 2047\b"):
        g.init_macros(None, ux)
    g.init_macros()  # defaults are valid; the handle still steps
    g.step(2, 1)


def test_many_cylinders_fp64_matches_oracle():
    """24 cylinders (1,224 markers): enough forced nodes that the one-launch
    step runs its IB sub-step in more than the minimum 8 blocks.  Fields and
    per-body forces against the oracle."""
    from ippi_lbm.validation import seeded_cylinders

    nx, ny, d = 640, 320, 16
    o, g = pair(nx, ny, collision=ip.MRT, bc_set=ip.BC_CHANNEL, u_in=0.05, tau0=0.56, cs=0.1,
                delta_kernel=ip.DELTA_PESKIN4, mdf_iters=2)
    cs = seeded_cylinders(nx, ny, d, 24, d, seed=3)
    nm = int(np.ceil(np.pi * d))
    xy = np.concatenate([cylinder_markers(cx, cy, d / 2, nm) for cx, cy in cs])
    body = np.repeat(np.arange(len(cs), dtype=np.int32), nm)
    ds = np.full(len(body), np.pi * d / nm)
    # forced nodes: every node within the 4 x 4 Peskin support of a marker
    forced = set()
    for x, y in xy:
        for i in range(int(np.floor(x)) - 1, int(np.floor(x)) + 3):
            for j in range(int(np.floor(y)) - 1, int(np.floor(y)) + 3):
                forced.add((i, j))
    assert len(forced) > 8 * 512
    o.set_markers(xy, body=body, ds=ds)
    g.set_markers(xy, body=body, ds=ds)
    y = np.arange(ny) + 0.5
    ux = np.tile((4 * 0.05 * y * (ny - y) / ny ** 2)[:, None], (1, nx))
    ux = ux + np.random.default_rng(1).uniform(-1e-4, 1e-4, ux.shape)
    o.init_macros(np.ones((ny, nx)), ux, np.zeros((ny, nx)))
    g.init_macros(np.ones((ny, nx)), ux, np.zeros((ny, nx)))
    for n, t0 in ((1, 1), (24, 2)):
        o.step(n, t0)
        g.step(n, t0)
        compare(o, g, 1e-11)
        fo, _ = o.forces()
        fg = g.forces()
        np.testing.assert_allclose(np.asarray(fg).reshape(-1), np.asarray(fo).reshape(-1), rtol=1e-9, atol=1e-14)
