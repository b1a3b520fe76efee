"""The alternative LES closures on the GPU (IPPI_LES_WALE, IPPI_LES_CSM,
IPPI_LES_DYNAMIC) against the FP64 oracle, in a channel with an IB cylinder
and a solid block, so that the velocity gradients meet IB-corrected nodes,
a solid, the walls and the outlet column.  FP64 storage to 1e-11 (the
populations, moments and the relaxation time of the next collision); FP32
storage against FP64 after 400 steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402
from ippi_lbm import scenes  # noqa: E402

NX, NY, CX, CY, D = 300, 64, 60.3, 31.7, 10


def params(coll, les, storage=ip.F64):
    return dict(collision=coll, storage=storage, bc_set=ip.BC_CHANNEL, les_model=les, tau0=0.56, cs=0.1,
                u_in=0.05, rho0=1.0, delta_kernel=ip.DELTA_PESKIN4, mdf_iters=1)


def scene(x, les):
    m = np.zeros((NY, NX), np.uint8)
    m[20:31, 200:211] = 1
    x.set_solid(m)
    xy, ds = scenes.cylinder_markers(CX, CY, D)
    x.set_markers(xy, ds=ds)
    if les == ip.LES_DYNAMIC:
        yy, xx = np.mgrid[0:NY, 0:NX].astype(float)
        x.set_wall_distance(np.hypot(xx - CX, yy - CY) - D / 2)
    x.init_macros(*scenes.channel_init(NX, NY, 0.05))


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("les", [ip.LES_WALE, ip.LES_CSM, ip.LES_DYNAMIC])
@pytest.mark.parametrize("coll", [ip.BGK, ip.MRT, ip.RR])
def test_closure_matches_oracle_fp64(coll, les):
    p = params(coll, les)
    g = ip.Lattice(NX, NY, **p)
    o = po.Oracle(NX, NY, collision=coll, bc_set=po.BC_CHANNEL, les_model=les, tau0=0.56, cs=0.1,
                  u_in=0.05, delta_kernel=ip.DELTA_PESKIN4, mdf_iters=1)
    scene(g, les)
    scene(o, les)
    t = 0
    for n in (1, 9, 40):
        assert o.step(n, t + 1) == 0
        g.step(n, t + 1)
        t += n
        for fg, fo in ((ip.FIELD_F, po.F), (ip.FIELD_RHO, po.RHO), (ip.FIELD_UX, po.UX),
                       (ip.FIELD_UY, po.UY), (ip.FIELD_TAU, po.TAU)):
            a, b = g.download(fg), o.get(fo)
            assert rel(a, b) < 1e-11, (t, fg, np.unravel_index(np.argmax(np.abs(a - b)), a.shape))
        np.testing.assert_allclose(g.forces().reshape(-1), np.asarray(o.forces()[0]).reshape(-1),
                                   rtol=1e-10, atol=1e-14)
    tau = g.download(ip.FIELD_TAU)
    assert (tau - 0.56).max() > 1e-6  # the closure is active
    g.close()


@pytest.mark.parametrize("les", [ip.LES_WALE, ip.LES_CSM, ip.LES_DYNAMIC])
def test_closure_fp32_against_fp64(les):
    out = {}
    for st in (ip.F64, ip.F32):
        g = ip.Lattice(NX, NY, **params(ip.MRT, les, st))
        scene(g, les)
        g.step(400, 1)
        out[st] = (g.download(ip.FIELD_UX), g.download(ip.FIELD_TAU), g.forces().reshape(-1))
        g.close()
    assert rel(out[ip.F32][0], out[ip.F64][0]) < 1e-4
    assert np.abs(out[ip.F32][1] - out[ip.F64][1]).max() < 1e-4
    np.testing.assert_allclose(out[ip.F32][2], out[ip.F64][2], rtol=1e-3, atol=1e-6)


def test_closure_argument_checks():
    with pytest.raises(ip.IppiError, match="channel"):
        ip.Lattice(64, 32, les_model=ip.LES_WALE)  # flat-plate scene
    g = ip.Lattice(64, 32, **params(ip.MRT, ip.LES_DYNAMIC))
    with pytest.raises(ip.IppiError, match="wall distance"):
        g.step(1, 1)
    g.set_wall_distance(np.full((32, 64), 5.0))
    g.step(2, 1)
    with pytest.raises(ip.IppiError, match="relaxation-time models"):
        g.adjoint_forward(4, 3, 2)
    with pytest.raises(ip.IppiError):
        g.set_wall_distance(np.full((32, 64), np.nan))
    g.close()


def test_driver_dynamic_closure_matches_api(tmp_path):
    """ippi_main --les dynamic: Mesh::SetNormalDis's distances (measured from
    the mirror index, x + 1 on one rank, as the reference does) reach the
    closure; the Tecplot fields equal the Python API's on the same lattice."""
    import os
    import subprocess

    from conftest import PKG_DIR

    nx, ny, u, re, cx, cy, d = 200, 64, 0.05, 100.0, 50.3, 32.1, 12.0
    r = subprocess.run([os.path.join(PKG_DIR, "ippi_main"), "--scene", "channel", "--nx", str(nx), "--ny",
                        str(ny), "--u", str(u), "--re", str(re), "--cs", "0.1", "--cylinder", str(cx), str(cy),
                        str(d), "--les", "dynamic", "--steps", "20", "--save", "20", "--print", "0"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    with open(tmp_path / "fluid" / "fluid_Merged_20.dat") as f:
        rows = np.array([[float(v) for v in ln.split()] for ln in f.read().splitlines()[3:] if ln.strip()])
    g = ip.Lattice(nx, ny, collision=ip.BGK, storage=ip.F64, bc_set=ip.BC_CHANNEL, les_model=ip.LES_DYNAMIC,
                   tau0=3.0 * (u * d / re) + 0.5, cs=0.1, u_in=u, rho0=1.0, delta_kernel=ip.DELTA_PESKIN4)
    yy, xx = np.mgrid[0:ny, 0:nx].astype(float)
    g.set_wall_distance(np.sqrt((xx + 1 - cx) ** 2 + (yy - cy) ** 2) - d / 2)
    xy, ds = scenes.cylinder_markers(cx, cy, d)
    g.set_markers(xy, ds=ds)
    g.init_macros()
    g.step(20, 1)
    for col, field in ((2, ip.FIELD_RHO), (3, ip.FIELD_UX), (4, ip.FIELD_UY), (7, ip.FIELD_TAU)):
        np.testing.assert_allclose(rows[:, col].reshape(nx, ny).T, g.download(field), rtol=1e-5, atol=1e-8)
    g.close()
