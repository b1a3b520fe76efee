"""The plain-method configuration run end to end on the GPU against the FP64
oracle: 400 x 100 channel, D = 20 cylinder at (100, 50) (63 markers, Peskin
4-point, direct forcing), parabolic Zou-He inlet u_max = 0.05, Re 100, BGK,
FP64, seeded +-1e-4 noise, 10,000 steps.  Drag / lift histories, the
Strouhal number, and the full population field at steps 100, 1000 and 10000
must agree with the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402
from ippi_lbm import learned_tau as lt  # noqa: E402
from ippi_lbm import scenes  # noqa: E402


def test_config1_cylinder_re100_matches_oracle():
    sc = scenes.config1()
    nx, ny, steps = sc["nx"], sc["ny"], 10000
    assert len(sc["ds"]) == 63
    p = sc["params"]
    g = ip.Lattice(nx, ny, **p)
    o = po.Oracle(nx, ny, collision=p["collision"], bc_set=po.BC_CHANNEL, les_model=p["les_model"],
                  tau0=p["tau0"], cs=p["cs"], u_in=p["u_in"], delta_kernel=p["delta_kernel"],
                  mdf_iters=p["mdf_iters"], avg_start=p["avg_start"])
    for x in (g, o):
        x.init_macros(*sc["init"])
        x.set_markers(sc["markers"], ds=sc["ds"])
    q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
    every = 10
    cd_o = np.zeros(steps // every)
    cl_o = np.zeros(steps // every)
    t = tg = 0
    for dump in (100, 1000, 10000):
        while t < dump:
            assert o.step(every, t + 1) == 0
            t += every
            f = np.asarray(o.forces()[0]).reshape(-1)
            cd_o[t // every - 1], cl_o[t // every - 1] = f[0] / q, f[1] / q
        g.step(dump - tg, tg + 1)
        tg = dump
        fo, fg = o.get(po.F), g.download(ip.FIELD_F)
        assert np.abs(fg - fo).max() / np.abs(fo).max() < 1e-10, dump
    hist = g.force_history(steps)[:, 0, :] / q
    cd_g, cl_g = hist[every - 1::every, 0], hist[every - 1::every, 1]
    np.testing.assert_allclose(cd_g, cd_o, rtol=1e-8, atol=1e-12)
    np.testing.assert_allclose(cl_g, cl_o, rtol=0, atol=1e-9)
    # periodic shedding: the Strouhal number of the second half of the run
    half = len(cl_o) // 2
    st_g = lt.strouhal(cl_g[half:], sc["d"], sc["u_ref"] * every)
    st_o = lt.strouhal(cl_o[half:], sc["d"], sc["u_ref"] * every)
    assert st_g == pytest.approx(st_o, rel=1e-9)
    assert 0.1 < lt.strouhal(hist[steps // 2:, 1], sc["d"], sc["u_ref"]) < 0.4
    cd_mean = hist[steps // 2:, 0].mean()
    assert 1.0 < cd_mean < 5.0, cd_mean


def test_config1_fp32_matches_fp64_drag_and_strouhal():
    """The same channel (Re 100, periodic shedding) with FP32 arithmetic on
    shifted populations against FP64: over the last 15,000 of 30,000 steps
    the mean drag, the lift amplitude and the Strouhal number agree within
    the 0.5 % the method states."""
    out = {}
    steps = 30000
    for st in (ip.F64, ip.F32):
        sc = scenes.config1()
        g = ip.Lattice(sc["nx"], sc["ny"], **dict(sc["params"], storage=st))
        g.init_macros(*sc["init"])
        g.set_markers(sc["markers"], ds=sc["ds"])
        g.step(steps, 1)
        q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
        h = g.force_history(steps // 2)[:, 0, :] / q
        out[st] = (h[:, 0].mean(), h[:, 1].std(), lt.strouhal(h[:, 1], sc["d"], sc["u_ref"]))
        g.close()
    (cd64, cl64, st64), (cd32, cl32, st32) = out[ip.F64], out[ip.F32]
    print(f"Cd {cd64:.6f} / {cd32:.6f}, Cl rms {cl64:.6f} / {cl32:.6f}, St {st64:.5f} / {st32:.5f}")
    assert 0.1 < st64 < 0.4 and cl64 > 1e-3  # shedding developed
    assert cd32 == pytest.approx(cd64, rel=5e-3)
    assert cl32 == pytest.approx(cl64, rel=5e-3)
    assert st32 == pytest.approx(st64, rel=5e-3)
