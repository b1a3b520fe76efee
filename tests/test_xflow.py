"""The XFlow import of the host layer (host/xflow.cpp; Mesh::ReadXflowdata,
ManageDataFromXflow, XflowABS, ChangeTauFromXflow, FindAndWriteTau,
mesh.cpp:2189-2766) against the restatement in oracle/xflow_ref.py: parse
rules, unit conversions, the merge of repeated points, clipping and node
matching bit for bit on CPU; on the GPU, the driver's --xflow-init /
--xflow-abs runs and the Mesh's tau methods against the Python API on the
same lattice."""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

import xflow_ref
from conftest import PKG_DIR, REPO

HOST = os.path.join(PKG_DIR, "host")
MAIN = os.path.join(PKG_DIR, "ippi_main")
HEADER = "id,x,y,z,VelocityModule,StaticPressure,Vort,TotalPressure,Turbulence,viscosity,Vx,Vy,Vz,Vmag"


def synth_csv(path, nx, ny, seed=0, block=(10, 21, 5, 16), nu0=0.02):
    """Points on nodes x0..x1-1, y0..y1-1 (jittered by < 5e-4 m, so they
    round onto the node), some repeated, a few lines the parser must skip,
    and points off the lattice."""
    rng = np.random.default_rng(seed)
    x0, x1, y0, y1 = block
    lines = [HEADER]
    k = 0

    def line(xm, ym, rho, ux, uy, nu):
        nonlocal k
        k += 1
        sp = (rho - 1.0) * 101325.0
        c = 340.112 * math.sqrt(3.0)
        vals = [k, xm, ym, 0.0, math.hypot(ux, uy) * c, sp, 0.0, 0.0, 0.0, nu, ux * c, uy * c, 0.0,
                math.hypot(ux, uy) * c]
        return ",".join(repr(float(v)) for v in vals)

    for x in range(x0, x1):
        for y in range(y0, y1):
            for _ in range(1 + (rng.random() < 0.3)):  # about 30 % repeated
                xm = x * 0.001 - 0.4 + rng.uniform(-4e-4, 4e-4)
                ym = y * 0.001 + rng.uniform(-4e-4, 4e-4)
                lines.append(line(xm, ym, 1 + rng.normal(0, 2e-3), 0.03 + rng.normal(0, 5e-3),
                                  rng.normal(0, 5e-3), nu0 + rng.uniform(0, 0.01)))
    lines.append("1,2,3")                      # short: skipped
    lines.append("a,b,c,d,e,f,g,h,i,j,k,l,m,n")  # not numbers: skipped
    lines.append(line(nx * 0.001 + 0.0, 0.003, 1, 0, 0, 0.02))      # beyond the outlet: clipped
    lines.append(line((nx - 1) * 0.001 - 0.4, (ny + 3) * 0.001, 1, 0, 0, 0.02))  # above the lattice
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


@pytest.fixture(scope="module")
def dump_bin(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("xflow") / "xflow_dump")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", HOST, os.path.join(HOST, "xflow.cpp"),
                    os.path.join(REPO, "tests", "xflow_dump.cpp"), "-o", out], check=True)
    return out


def test_reader_matches_restatement(dump_bin, tmp_path):
    nx, ny = 64, 32
    path = str(tmp_path / "pb_1.csv")
    synth_csv(path, nx, ny)
    r = subprocess.run([dump_bin, path, str(nx), str(ny)], capture_output=True, text=True, check=True)
    got = [ln.split() for ln in r.stdout.splitlines()]
    want = xflow_ref.clip(xflow_ref.read(path), nx)
    assert len(got) == len(want) == 11 * 11 + 1  # the block, and the point above the lattice
    for g, w in zip(got, want):
        vals = [float(v) for v in g[:10]]
        ref = [w[k] for k in ("vx", "vy", "vz", "VelocityModule", "StaticPress", "TotalPressure",
                              "viscosity", "ux", "uy", "uz")]
        assert vals == ref  # bit for bit (printed with 17 digits)
        node = xflow_ref.node_of(w, nx, ny)
        assert (int(g[10]), int(g[11])) == (node if node else (-1, -1))
    # every block node is hit exactly once
    nodes = {xflow_ref.node_of(w, nx, ny) for w in want} - {None}
    assert nodes == {(x, y) for x in range(10, 21) for y in range(5, 16)}


def test_reader_rejects_missing_file(dump_bin, tmp_path):
    r = subprocess.run([dump_bin, str(tmp_path / "none.csv"), "8", "8"], capture_output=True)
    assert r.returncode == 1


def read_tecplot(path):
    with open(path) as f:
        lines = f.read().splitlines()
    return np.array([[float(v) for v in ln.split()] for ln in lines[3:] if ln.strip()])


def columns(rows, nx, ny):
    """Density, U, V of a WriteDatFluid file as [ny][nx] planes (x-major rows)."""
    return [rows[:, c].reshape(nx, ny).T for c in (2, 3, 4)]


@pytest.mark.gpu
def test_driver_xflow_init_and_abs_match_api(tmp_path):
    ip = pytest.importorskip("ippi_lbm")
    nx, ny, u, re, offset = 64, 32, 0.05, 100.0, 7
    d = tmp_path / "xf"
    d.mkdir()
    for t in (1, 2, 3, 4):
        synth_csv(str(d / f"pb_{t + offset}.csv"), nx, ny, seed=t)
    run = tmp_path / "run"
    run.mkdir()
    r = subprocess.run([MAIN, "--scene", "channel", "--nx", str(nx), "--ny", str(ny), "--u", str(u),
                        "--re", str(re), "--steps", "4", "--save", "1", "--print", "0",
                        "--xflow", str(d), "--xflow-offset", str(offset), "--xflow-init",
                        "--xflow-abs", "3"], cwd=run, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]

    g = ip.Lattice(nx, ny, collision=ip.BGK, storage=ip.F64, bc_set=ip.BC_CHANNEL,
                   les_model=ip.LES_SMAGORINSKY, tau0=0.5 + 6.0 * ((ny * u) / re), cs=0.173, u_in=u,
                   rho0=1.0, delta_kernel=ip.DELTA_PESKIN4)
    g.init_macros()
    want = {}
    for t in (1, 2, 3, 4):
        g.step(1, t)
        m = [g.download(k) for k in (ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY)]
        if t == 1:  # ManageDataFromXflow: imported moments, then equilibrium everywhere
            for p in xflow_ref.clip(xflow_ref.read(str(d / f"pb_{1 + offset}.csv")), nx):
                node = xflow_ref.node_of(p, nx, ny)
                if node:
                    x, y = node
                    m[0][y, x], m[1][y, x], m[2][y, x] = p["TotalPressure"], p["ux"], p["uy"]
            g.reequilibrate(*m)
        if t == 3:  # XflowABS: equilibrium of the current moments everywhere
            g.reequilibrate(*m)
        want[t] = m
    for t in (1, 2, 3, 4):
        got = columns(read_tecplot(run / "fluid" / f"fluid_Merged_{t}.dat"), nx, ny)
        for a, b in zip(got, want[t]):
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-8)
    # the imported density differs from the solver's: the reset is visible
    assert np.abs(want[1][0] - 1.0).max() > 1e-3
    g.close()


def change_tau(points, nx, ny, rho, ux, uy, tau0):
    """ChangeTauFromXflow's restatement (host/mesh.cpp): x-major visit, the
    last matched point's viscosity and errors carried into nodes no point
    lands on, starting from nu = (tau0 - 1/2) / 3 and zero errors."""
    at = {}
    for q, p in enumerate(points):
        node = xflow_ref.node_of(p, nx, ny)
        if node:
            at[node] = q
    nu = (tau0 - 0.5) / 3.0
    ev = er = tv = tr = 0.0
    tau = np.zeros((ny, nx))
    for x in range(nx):
        for y in range(ny):
            if (x, y) in at:
                p = points[at[(x, y)]]
                nu = p["viscosity"]
                ev = (ux[y, x] - p["ux"]) * (ux[y, x] - p["ux"]) + (uy[y, x] - p["uy"]) * (uy[y, x] - p["uy"])
                er = (rho[y, x] - p["TotalPressure"]) * (rho[y, x] - p["TotalPressure"])
            tv += ev
            tr += er
            tau[y, x] = 0.5 + 3.0 * nu
    return tau, tv / (nx * ny), tr / (nx * ny)


@pytest.mark.gpu
def test_mesh_change_tau_and_find_and_write_tau(tmp_path):
    ip = pytest.importorskip("ippi_lbm")
    cxx = shutil.which("g++") or shutil.which("c++")
    nx, ny, offset, X, Y = 64, 32, 5, 15, 10
    d = tmp_path / "xf"
    d.mkdir()
    for t in (1, 2, 3):
        # tau = 1/2 + 3 nu >= 0.71: the scan's dtau >= -0.1 keeps it above 1/2
        synth_csv(str(d / f"pb_{t + offset}.csv"), nx, ny, seed=10 + t, nu0=0.07)
    exe = str(tmp_path / "xflow_mesh")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", HOST, "-I", os.path.join(REPO, "include"),
                    os.path.join(HOST, "mesh.cpp"), os.path.join(HOST, "NodeAndLattice.cpp"),
                    os.path.join(HOST, "xflow.cpp"), os.path.join(REPO, "tests", "xflow_mesh.cpp"),
                    "-o", exe, "-L", PKG_DIR, "-lippi_lbm", "-Wl,-rpath," + PKG_DIR], check=True)
    run = tmp_path / "run"
    run.mkdir()
    r = subprocess.run([exe, str(d), str(offset), str(nx), str(ny), str(X), str(Y)], cwd=run,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]

    g = ip.Lattice(nx, ny, collision=ip.BGK, storage=ip.F64, bc_set=ip.BC_CHANNEL,
                   les_model=ip.LES_FIELD, tau0=0.76, cs=0.1, u_in=0.05, rho0=1.0)
    g.set_tau_field(np.full((ny, nx), 0.76))
    g.init_macros()
    pts = xflow_ref.clip(xflow_ref.read(str(d / f"pb_{1 + offset}.csv")), nx)
    m = [g.download(k) for k in (ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY)]
    tau, mse_v, mse_r = change_tau(pts, nx, ny, *m, 0.76)
    line = np.loadtxt(run / "cp" / "InletMSE.dat")
    assert line[0] == 1
    np.testing.assert_allclose(line[1:], [mse_v, mse_r], rtol=1e-5)
    g.set_tau_field(tau)
    g.step(2, 1)
    tgt = None
    for p in xflow_ref.clip(xflow_ref.read(str(d / f"pb_{3 + offset}.csv")), nx):
        if xflow_ref.node_of(p, nx, ny) == (X, Y):
            tgt = [p["TotalPressure"], p["ux"], p["uy"]]
    best, _ = g.tau_scan([[X, Y]], [tgt])
    row = np.loadtxt(run / "cp" / "BestTau.dat")
    assert row[0] == 2
    assert abs(row[1] - best[0]) < 1e-12
    for ex, ey in [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)]:
        tau[Y + ey, X + ex] += best[0]
    np.testing.assert_allclose(row[2:], [tau[Y + ey, X + ex] for ex, ey in
                                         [(0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1),
                                          (-1, -1), (1, -1)]], rtol=1e-5)
    g.set_tau_field(tau)
    g.step(1, 3)
    got = columns(read_tecplot(run / "fluid" / "fluid_Merged_3.dat"), nx, ny)
    for a, b in zip(got, [g.download(k) for k in (ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY)]):
        np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-8)
    g.close()
