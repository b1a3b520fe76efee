"""The reference Mesh methods that the fused GPU step absorbs or that act on
the host mirror (host/mesh.h; reference mesh.h:52-107), through a C++
harness (tests/mesh_api.cpp) built against the host layer and the library.

CPU: Peskin's kernel DiracDelta against the formula of mesh.cpp:1354-1385,
the distance helpers, isAvailable, FilterLBM, and the refusal of the
sub-steps OneLBMStep fuses (message, errorflag, nothing changed).
GPU: OneLBMStep's per-call Cs reaches the device (tau equal to a Python
lattice run with that Cs), CaculateLESTau on the mirror equals the device's
Smagorinsky tau, NNmodel_Type0x reports loaded and absent nets,
InterpolateVel / CalParticleForce restated in numpy from the same velocity
field, and UpdateBoundary moves the markers the GPU step then uses.
"""
import math
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, PKG_DIR, REPO

HOST = os.path.join(PKG_DIR, "host")
LIB = os.path.join(PKG_DIR, "libippi_lbm.so")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx or not os.path.exists(LIB):
        pytest.skip("no C++ compiler or library not built")
    out = str(tmp_path_factory.mktemp("mesh_api") / "mesh_api")
    srcs = [os.path.join(HOST, f) for f in ("mesh.cpp", "NodeAndLattice.cpp", "xflow.cpp")]
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(REPO, "include"), "-I", HOST, *srcs,
                    os.path.join(REPO, "tests", "mesh_api.cpp"), "-o", out, "-L", PKG_DIR, "-lippi_lbm",
                    f"-Wl,-rpath,{PKG_DIR}"], check=True)
    return out


def parse(text):
    out = {}
    for ln in text.splitlines():
        p = ln.split()
        if p:
            out.setdefault(p[0], []).append(p[1:])
    return out


def peskin(x):
    a = abs(x)
    if a < 1:
        return (3 - 2 * a + math.sqrt(1 + 4 * a - 4 * x * x)) / 8
    if a < 2:
        return (5 - 2 * a - math.sqrt(-7 + 12 * a - 4 * x * x)) / 8
    return 0.0


def test_helpers_and_refusals(harness):
    r = subprocess.run([harness, "cpu"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    o = parse(r.stdout)
    for x, v in o["delta"]:
        assert float(v) == pytest.approx(peskin(float(x)), abs=1e-15)
    assert float(o["delta2"][0][0]) == pytest.approx(peskin(0.3) * peskin(-1.2), abs=1e-15)
    assert float(o["dis"][0][0]) == 5.0
    assert float(o["linedist"][0][0]) == 4.0  # centre (3, 4) to the x axis
    assert float(o["pointdist"][0][0]) == 5.0
    assert o["available_empty"][0][0] == "0"
    assert o["errorflag_before"][0][0] == "0" and o["errorflag_after"][0][0] == "1"
    assert o["errorflag_all"][0][0] == "1"
    assert o["nn_unloaded"][0][0] == "-1"
    for name in ("Streaming", "BoundaryCondition", "SpreadForce", "UpdateVelocity", "XflowBoundary"):
        assert f"Mesh::{name}:" in r.stderr


@pytest.mark.gpu
def test_per_call_cs_les_tau_nets_and_markers(harness, tmp_path):
    ip = pytest.importorskip("ippi_lbm")
    r = subprocess.run([harness, "gpu", os.path.join(GOLDEN, "band_nets")], capture_output=True, text=True,
                       timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stderr
    o = parse(r.stdout)

    # per-call Cs: steps 1-3 with 0.173, 4-6 with 0.3, as a Python lattice does
    g = ip.Lattice(416, 24, storage=ip.F64, tau0=0.52, cs=0.173)
    g.load_band_net(3, np.fromfile(os.path.join(GOLDEN, "band_nets", "AutoT03.f32"), dtype=np.float32))
    g.step(3, 1)
    g.set_les_cs(0.3)
    g.step(3, 4)
    tau = g.download(ip.FIELD_TAU)
    dev = float(o["device_tau"][0][0])
    assert dev == tau[10, 200]
    # CaculateLESTau on the mirror (FP64 host arithmetic) = the device's Smagorinsky tau
    assert float(o["host_tau"][0][0]) == pytest.approx(dev, rel=1e-13)
    assert o["nn03"][0][0] == "0" and o["nn01"][0][0] == "-1"
    assert int(o["nnflags_row22"][0][0]) == int(g.download(ip.FIELD_NNFLAG)[22].sum()) > 0

    # InterpolateVel / CalParticleForce against numpy on the same velocity field
    u = np.loadtxt(tmp_path / "u_field.txt").reshape(48, 160, 2)
    for q, x, y, vx, vy, fx, fy in o["marker"]:
        x, y = float(x), float(y)
        xi, yi = int(x), int(y)
        wx = wy = 0.0
        for X in range(xi - 1, xi + 3):
            for Y in range(yi - 1, yi + 3):
                w = peskin(x - X) * peskin(y - Y)
                wx += u[Y, X, 0] * w
                wy += u[Y, X, 1] * w
        assert float(vx) == pytest.approx(wx, abs=1e-14)
        assert float(vy) == pytest.approx(wy, abs=1e-14)
        assert float(fx) == pytest.approx(-2 * wx, abs=1e-14)  # prescribed velocity 0
        assert float(fy) == pytest.approx(-2 * wy, abs=1e-14)
    moved, want = map(float, o["moved"][0])
    assert moved == want
    assert o["errorflag"][0][0] == "0"
