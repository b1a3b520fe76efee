"""The precision sweep's storage modes against the FP64 CPU oracle on a crop
of the same geometry.

The sweep lattice (16384 x 4096, 64 seeded cylinders D = 48, Re 1000, MRT +
Smagorinsky) is too large for the CPU oracle, so its comparison runs on a
2048 x 512 window of the same layout (validation.config3_crop_scene: the
window with the most whole cylinders, here 4, as a channel of its own).  The
oracle runs that crop in FP64; the GPU runs it with FP32, FP16 and BF16
population storage (FP32 arithmetic).  Over `steps` steps, with statistics
over the last `avg`:

* per-cylinder mean drag coefficient, relative to the oracle's;
* L2 of the time-averaged velocity field, relative to the oracle's;
* mass drift (m_end - m_start) / m_start, against the oracle's.

Tolerances (stated per storage): FP32 Cd 1e-4, velocity L2 1e-4, mass drift
within 1e-7 of the oracle's; FP16 Cd 1 %, L2 1 %; BF16 Cd 10 %, L2 5 %,
drifts within 1e-3.

    python tests/test_config3_crop_gpu.py [--steps N] [--avg M]
prints the same comparison as one JSON line.
"""
import json
import os
import sys
import time

import numpy as np
import pytest

if __name__ == "__main__":
    sys.path[:0] = [os.path.dirname(os.path.abspath(__file__))]
    import conftest  # noqa: F401  (repository paths)

import pyoracle as po  # noqa: E402

TOL = {"f32": dict(cd=1e-4, l2=1e-4, drift=1e-7), "f16": dict(cd=1e-2, l2=1e-2, drift=1e-3),
       "bf16": dict(cd=1e-1, l2=5e-2, drift=1e-3)}


def crop_compare(steps=2000, avg=1000, storages=("f32", "f16", "bf16")):
    import ippi_lbm as ip
    from ippi_lbm.validation import config3_crop_scene

    st_of = {"f32": ip.F32, "f16": ip.F16, "bf16": ip.BF16}
    sc = config3_crop_scene()
    nx, ny = sc["nx"], sc["ny"]
    nb = len(sc["centres"])
    q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
    avg_from = steps - avg + 1

    po.build_oracle()
    p = dict(sc["params"], avg_start=avg_from)
    p.pop("storage")
    o = po.Oracle(nx, ny, **p)
    o.init_macros(*sc["init"])
    o.set_markers(sc["markers"], ds=sc["ds"], body=sc["bodies"])
    m0 = o.forces()[1]
    cd = np.zeros((steps, nb))
    t0 = time.perf_counter()
    for t in range(1, steps + 1):
        assert o.step(1, t) == 0
        cd[t - 1] = o.forces()[0][:, 0] / q
    oracle_s = time.perf_counter() - t0
    ref = dict(cd=cd[steps - avg:].mean(0), drift=(o.forces()[1] - m0) / m0,
               avg=np.stack([o.get(po.AVG_U), o.get(po.AVG_V)]))
    out = dict(window=[int(v) for v in sc["window"]], nx=nx, ny=ny, cylinders=nb, steps=steps, avg=avg,
               oracle_threads=po.threads(), oracle_s=round(oracle_s, 1),
               f64_cd=[round(float(v), 6) for v in ref["cd"]], f64_mass_drift=float(ref["drift"]))
    for name in storages:
        g = ip.Lattice(nx, ny, **dict(sc["params"], storage=st_of[name], avg_start=avg_from))
        g.init_macros(*sc["init"])
        g.set_markers(sc["markers"], ds=sc["ds"], body=sc["bodies"])
        _, gm0 = g.forces(with_mass=True)
        g.step(steps, 1)
        f = g.force_history(steps)
        _, gm1 = g.forces(with_mass=True)
        gavg = np.stack([g.download(ip.FIELD_AVG_U), g.download(ip.FIELD_AVG_V)])
        g.close()
        gcd = f[steps - avg:, :, 0].mean(0) / q
        rel = np.abs(gcd - ref["cd"]) / np.abs(ref["cd"])
        l2 = float(np.sqrt(np.sum((gavg - ref["avg"]) ** 2) / np.sum(ref["avg"] ** 2)))
        out[name] = dict(cd_rel_err_max=float(rel.max()), cd_rel_err_mean=float(rel.mean()),
                         mean_velocity_l2=l2, mass_drift=float((gm1 - gm0) / gm0))
    return out


@pytest.mark.gpu
def test_crop_storage_modes_against_the_oracle():
    pytest.importorskip("ippi_lbm")
    r = crop_compare()
    print(json.dumps(r))
    assert r["cylinders"] >= 3
    for name, tol in TOL.items():
        s = r[name]
        assert s["cd_rel_err_max"] <= tol["cd"], (name, s)
        assert s["mean_velocity_l2"] <= tol["l2"], (name, s)
        assert abs(s["mass_drift"] - r["f64_mass_drift"]) <= tol["drift"], (name, s, r["f64_mass_drift"])


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--avg", type=int, default=1000)
    a = ap.parse_args()
    print(json.dumps(crop_compare(a.steps, a.avg)), flush=True)
