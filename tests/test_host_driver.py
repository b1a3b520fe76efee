"""The C++ host layer (host/: Mesh, Lattice and the main.cpp driver over the
C ABI).  The driver's Tecplot output must hold the oracle's fields (to the
6 significant digits the reference's writer prints), per-step and batched
driving must give the same forces, and the driver must build without a GPU.
"""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_DIR

MAIN = os.path.join(PKG_DIR, "ippi_main")


def run_main(args, cwd, timeout=300):
    r = subprocess.run([MAIN, *args], cwd=cwd, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def read_tecplot(path):
    """Rows of a WriteDatFluid file (three header lines, then X Y values)."""
    with open(path) as f:
        lines = f.read().splitlines()
    assert lines[0].startswith("TITLE") and lines[1].startswith("VARIABLES")
    return np.array([[float(v) for v in ln.split()] for ln in lines[3:] if ln.strip()])


def test_driver_builds_and_prints_usage():
    assert os.path.exists(MAIN), "build.py builds ippi_main"
    r = subprocess.run([MAIN, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage: ippi_main" in r.stderr


@pytest.mark.gpu
def test_driver_plate_output_matches_oracle(tmp_path):
    import pyoracle as po

    nx, ny, steps, save, avg = 416, 12, 30, 10, 15
    re, u, cs = 5e5, 0.1, 0.173
    run_main(["--scene", "plate", "--nx", str(nx), "--ny", str(ny), "--steps", str(steps),
              "--save", str(save), "--avg", str(avg), "--print", "0"], cwd=tmp_path)
    tau0 = 0.5 + 6.0 * ((ny * u) / re)
    o = po.Oracle(nx, ny, collision=po.BGK, tau0=tau0, cs=cs, u_in=u, avg_start=avg)
    for t in range(1, steps + 1):
        o.step(1, t)
        if t % save:
            continue
        rows = read_tecplot(tmp_path / "fluid" / f"fluid_Merged_{t}.dat")
        assert rows.shape == (nx * ny, 9)
        # x-major: row = x * ny + y
        x, y = rows[:, 0].astype(int), rows[:, 1].astype(int)
        assert np.array_equal(x, np.repeat(np.arange(nx), ny))
        assert np.array_equal(y, np.tile(np.arange(ny), nx))
        want = {2: po.RHO, 3: po.UX, 4: po.UY, 5: po.AVG_U, 6: po.AVG_V, 7: po.TAU, 8: po.AVG_RHO}
        for col, fld in want.items():
            ref = o.get(fld).T.reshape(-1)  # [ny][nx] -> x-major
            scale = max(float(np.abs(ref).max()), 1e-30)
            err = float(np.abs(rows[:, col] - ref).max()) / scale
            assert err < 2e-5, (t, col, err)
        # the per-rank file is merged and removed
        assert not (tmp_path / "fluid" / f"fluid_t{t}_0.dat").exists()


@pytest.mark.gpu
def test_driver_channel_cylinder_batched_equals_per_step(tmp_path):
    common = ["--scene", "channel", "--nx", "200", "--ny", "64", "--u", "0.05", "--re", "100",
              "--cs", "0.1", "--cylinder", "50.3", "32.1", "12", "--steps", "60", "--save", "30",
              "--avg", "1000000", "--print", "0"]
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    run_main(common, cwd=a)
    run_main(common + ["--batched"], cwd=b)
    fa = np.loadtxt(a / "particle" / "forces.dat")
    fb = np.loadtxt(b / "particle" / "forces.dat")
    assert fa.shape == (60, 5) and np.array_equal(fa[:, 0], np.arange(1, 61))
    np.testing.assert_array_equal(fa, fb)
    # the cylinder holds the flow back: positive drag once the wake forms
    assert fa[-1, 3] > 0
    for t in (30, 60):
        np.testing.assert_array_equal(read_tecplot(a / "fluid" / f"fluid_Merged_{t}.dat"),
                                      read_tecplot(b / "fluid" / f"fluid_Merged_{t}.dat"))
    n = math.ceil(math.pi * 12)
    with open(a / "particle" / "particle_t0.dat") as f:
        assert f"N={n}, E={n}" in f.read()


@pytest.mark.gpu
def test_driver_solid_cylinder_cd_and_cp(tmp_path):
    """--solid: the cylinder as solid nodes, Mesh::OutputCd every step (every
    save point when batched) and the time-averaged Cp of its 'b' nodes; the
    values the driver prints (6 digits) are those of the Python API on the
    same lattice (the driver's defaults: BGK, FP64, Smagorinsky)."""
    ip = pytest.importorskip("ippi_lbm")
    from ippi_lbm import scenes

    nx, ny, u, d = 400, 100, 0.05, 20
    init = np.stack(scenes.channel_init(nx, ny, u))
    init.tofile(tmp_path / "init.f64")
    common = ["--scene", "channel", "--nx", str(nx), "--ny", str(ny), "--u", str(u), "--re", "100",
              "--cs", "0.1", "--cylinder", "100", "50", str(d), "--solid", "--steps", "2000", "--save", "1000",
              "--avg", "1000", "--cp", "1000", "--print", "0", "--init", str(tmp_path / "init.f64")]
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    run_main(common, cwd=a)
    run_main(common + ["--batched"], cwd=b)
    ca = np.loadtxt(a / "particle" / "CD_CL.dat")
    cb = np.loadtxt(b / "particle" / "CD_CL.dat")
    assert ca.shape == (2000, 3) and np.array_equal(ca[:, 0], np.arange(1, 2001))
    assert cb.shape == (2, 3)
    np.testing.assert_array_equal(ca[[999, 1999]], cb)
    assert 1.0 < ca[-500:, 1].mean() < 2.0
    assert not (a / "particle" / "forces.dat").exists()
    cp = np.loadtxt(a / "cp" / "cp_Merged_2000.dat")
    np.testing.assert_array_equal(cp, np.loadtxt(b / "cp" / "cp_Merged_2000.dat"))
    assert not (a / "cp" / "cp_2000_0.dat").exists()

    q = 0.5 * u * u * d
    g = ip.Lattice(nx, ny, collision=ip.BGK, storage=ip.F64, bc_set=ip.BC_CHANNEL,
                   les_model=ip.LES_SMAGORINSKY, tau0=3.0 * (u * d / 100) + 0.5, cs=0.1, u_in=u, rho0=1.0,
                   avg_start=1000)
    g.set_solid(scenes.cylinder_solid(nx, ny, 100, 50, d))
    g.init_macros(*init)
    for t, row in ((1, cb[0]), (1001, cb[1])):
        g.step(1000, t)
        np.testing.assert_allclose(g.solid_force() / q, row[1:], rtol=2e-5, atol=1e-6)
    # the 'b' ring around a D = 20 staircase cylinder (317 's' nodes): 88 nodes
    style = g.download(ip.FIELD_FLAGS)
    ys, xs = np.nonzero(style == ord("b"))
    assert len(cp) == 88 == len(xs)
    want = (g.download(ip.FIELD_AVG_RHO)[ys, xs] / 3 - 1 / 3) / (0.5 * u * u)
    order = np.lexsort((ys, xs))  # the driver writes x-major
    np.testing.assert_allclose(cp[:, 2], want[order], rtol=2e-5, atol=1e-6)
    front = cp[np.argmin(cp[:, 0])]
    assert front[2] > 0.5  # stagnation side
    assert cp[:, 2].min() < 0  # suction on the flanks
    g.close()


@pytest.mark.gpu
def test_driver_checkpoint_resume_and_metrics_log(tmp_path):
    """--checkpoint at the save points, --resume from the one at step 30:
    the resumed run writes the same fields and forces as the uninterrupted
    one; --metrics writes one JSON line per --print step."""
    import json
    import shutil

    common = ["--scene", "channel", "--nx", "200", "--ny", "64", "--u", "0.05", "--re", "100",
              "--cs", "0.1", "--cylinder", "50.3", "32.1", "12", "--steps", "60", "--save", "30",
              "--avg", "40", "--print", "10"]
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    run_main(common + ["--checkpoint", "state30.ippi", "--steps", "30", "--metrics", "m.jsonl"], cwd=a)
    shutil.copy(a / "state30.ippi", b / "state30.ippi")
    run_main(common + ["--checkpoint", "state.ippi"], cwd=a)
    out = run_main(common + ["--resume", "state30.ippi", "--checkpoint", "state.ippi"], cwd=b)
    assert "Resumed at step 31" in out
    fa = np.loadtxt(a / "particle" / "forces.dat")
    fb = np.loadtxt(b / "particle" / "forces.dat")
    assert fa.shape == (90, 5) and fb.shape == (30, 5)  # run a wrote 30 + 60 lines
    np.testing.assert_array_equal(fa[-30:], fb)
    np.testing.assert_array_equal(read_tecplot(a / "fluid" / "fluid_Merged_60.dat"),
                                  read_tecplot(b / "fluid" / "fluid_Merged_60.dat"))
    assert (a / "state.ippi").read_bytes() == (b / "state.ippi").read_bytes()
    rows = [json.loads(ln) for ln in (a / "m.jsonl").read_text().splitlines()]
    assert [r["step"] for r in rows] == [10, 20, 30]
    for r in rows:
        assert r["mlups"] > 0 and r["hbm_gbs"] == pytest.approx(r["mlups"] * 0.144)
        # FP64 mass of the open channel (Zou-He inflow, NEE outflow): near rho0 per node
        assert abs(r["mass"] / (200 * 64) - 1) < 0.01 and 0.04 < r["max_u"] < 0.2
        assert math.isfinite(r["cd"]) and math.isfinite(r["cl"])
        assert r["tau_net_nodes"] == 0 and r["tau_fallback_nodes"] == 0
