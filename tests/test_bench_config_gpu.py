"""Step-level parity of the benchmarked configuration itself with the FP64 oracle.

The bench line is measured on the 4096 x 1024 channel with one immersed-
boundary cylinder (D = 128, 403 markers, Peskin 4-point delta, one direct-
forcing pass), Re 3900, MRT + Smagorinsky Cs 0.1, FP32 storage and FP32
arithmetic with the hardware reciprocal and square root.  Here the same
lattice, markers and seeded initial fields go through the C ABI and through
the oracle (FP64, the reference's arithmetic), and after 1 and after 11 steps:

* populations, rho and u agree to 1e-5 (1 step) and 1e-4 (11 steps) relative
  to each field's scale (max |f|, 1, max |u_x|), the tolerance the method
  states for FP32;
* the FP64 body force on the cylinder agrees to the same relative tolerance
  of |F|, and the FP64 mass to 1e-7.

The same is checked for the RR operator, the configuration's second run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402
from ippi_lbm import scenes  # noqa: E402


def field_errors(o, g):
    uscale = max(float(np.abs(o.get(po.UX)).max()), 1e-12)
    out = {}
    for name, fo, fg, scale in (("f", po.F, ip.FIELD_F, None), ("rho", po.RHO, ip.FIELD_RHO, 1.0),
                                ("ux", po.UX, ip.FIELD_UX, uscale), ("uy", po.UY, ip.FIELD_UY, uscale)):
        b = o.get(fo)
        a = g.download(fg)
        s = float(np.abs(b).max()) if scale is None else scale
        out[name] = float(np.abs(a - b).max()) / s
        del a, b
    return out


@pytest.mark.parametrize("coll", [ip.MRT, ip.RR])
def test_bench_configuration_matches_oracle(oracle, coll):
    oracle.build_oracle()
    sc = scenes.config2(collision=coll)
    nx, ny = sc["nx"], sc["ny"]
    assert (nx, ny) == (4096, 1024) and len(sc["ds"]) == 403
    p = dict(sc["params"])
    assert p["storage"] == ip.F32 and p["les_model"] == ip.LES_SMAGORINSKY and p["cs"] == 0.1
    g = ip.Lattice(nx, ny, **p)
    p.pop("storage")
    o = po.Oracle(nx, ny, **p)
    for x in (g, o):
        x.init_macros(*sc["init"])
        x.set_markers(sc["markers"], ds=sc["ds"])
    t = 1
    for n, tol in ((1, 1e-5), (10, 1e-4)):
        assert o.step(n, t) == 0
        g.step(n, t)
        t += n
        err = field_errors(o, g)
        assert max(err.values()) <= tol, (t - 1, err)
        fo, mo = o.forces()
        fg, mg = g.forces(with_mass=True)
        assert np.abs(fg - fo).max() / np.abs(fo).max() <= tol, (fg, fo)
        assert abs(mg - mo) / mo <= 1e-7, (mg, mo)
    g.close()
