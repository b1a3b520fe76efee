"""The oracle is pinned before it is trusted.

* against the reference build (oracle/build_ref.sh, fixtures from
  tests/golden/make_golden.py): every field of the flat-plate step must be
  bit-identical (SHA-256 of the float64 arrays), for BGK, MRT and RR with the
  Smagorinsky tau, with and without the boundary nets, and the IB primitives
  (bilinear and Peskin) must match;
* against the shipped TorchScript boundary nets (outputs computed by torch);
* against analytic identities of the lattice-Boltzmann method.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

GOLD = json.load(open(os.path.join(GOLDEN, "ref_golden.json")))
NETS = np.load(os.path.join(GOLDEN, "band_net_golden.npz"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def load_net(t):
    return np.fromfile(os.path.join(GOLDEN, "band_nets", f"AutoT0{t}.f32"), dtype=np.float32)


@pytest.mark.parametrize("t", [1, 3, 5, 7])
def test_band_net_forward_matches_torch(oracle, t):
    """orc_band_forward == torch's forward of NNmodel/AutoT0t.pt (float32)."""
    import ctypes as C

    w = load_net(t)
    assert w.size == 101249
    x, y = NETS[f"x{t}"], NETS[f"y{t}"]
    L = oracle.lib()
    out = np.array([L.orc_band_forward(w.ctypes.data_as(C.POINTER(C.c_float)), 15,
                                       np.ascontiguousarray(xi).ctypes.data_as(C.POINTER(C.c_float)))
                    for xi in x], np.float32)
    np.testing.assert_allclose(out, y, rtol=2e-6, atol=2e-6)


def test_band_net_known_values():
    """Outputs on (u=0.1, v=0, rho=1) x 5 quoted for the shipped nets."""
    for t, v in ((1, 0.50499), (3, 0.50797), (5, 0.51334), (7, 0.50066)):
        assert abs(float(NETS[f"y{t}"][0]) - v) < 1e-5


@pytest.mark.parametrize("name", sorted(GOLD["plate"]))
def test_oracle_bit_exact_with_reference_plate(oracle, name):
    g = GOLD["plate"][name]
    c = g["case"]
    coll = {"srt": oracle.BGK, "mrt": oracle.MRT, "rr": oracle.RR}[c["variant"]]
    o = oracle.Oracle(c["nx"], c["ny"], collision=coll, tau0=c["tau"], cs=c["cs"], u_in=0.1,
                      avg_start=c["avg_start"], plate_x0=400)
    if c["nets"]:
        for t in (1, 3, 5, 7):
            o.load_band_net(t, load_net(t))
    flags = o.get(oracle.FLAGS).astype(np.uint8)
    assert hashlib.sha256(flags.tobytes()).hexdigest() == g["flags_sha"]
    done = 0
    fields = {"F": oracle.F, "rho": oracle.RHO, "ux": oracle.UX, "uy": oracle.UY,
              "avg_u": oracle.AVG_U, "avg_v": oracle.AVG_V, "avg_rho": oracle.AVG_RHO}
    pts = g["sample_nodes"]
    for snap in g["snapshots"]:
        rc = o.step(snap["step"] - done, done + 1)
        done = snap["step"]
        assert rc == snap["rc"]
        for fname, fid in fields.items():
            a = o.get(fid)
            if fid == oracle.F:
                got = [[float(a[k, y, x]) for k in range(9)] for x, y in pts]
            else:
                got = [float(a[y, x]) for x, y in pts]
            assert got == snap["sample"][fname], fname
            assert sha(a) == snap["hash"][fname], fname


@pytest.mark.parametrize("name", sorted(GOLD["plate"]))
def test_oracle_next_tau_is_reference_tau_one_step_later(oracle, name):
    """The oracle's TAU is the relaxation time of the next collision; the
    reference's LatMesh tau after step n+1 is that same value."""
    g = GOLD["plate"][name]
    c = g["case"]
    coll = {"srt": oracle.BGK, "mrt": oracle.MRT, "rr": oracle.RR}[c["variant"]]
    o = oracle.Oracle(c["nx"], c["ny"], collision=coll, tau0=c["tau"], cs=c["cs"], u_in=0.1,
                      avg_start=c["avg_start"])
    if c["nets"]:
        for t in (1, 3, 5, 7):
            o.load_band_net(t, load_net(t))
    s0, s1 = g["snapshots"][0], g["snapshots"][1]
    o.step(s1["step"] - 1, 1)
    tau = o.get(oracle.TAU)
    flag = o.get(oracle.NNFLAG)
    pts = g["sample_nodes"]
    assert [float(tau[y, x]) for x, y in pts] == s1["sample"]["tau"]
    assert sha(tau) == s1["hash"]["tau"]
    assert sha(flag) == s1["hash"]["nnflag"]
    assert s0["step"] == 1


@pytest.mark.parametrize("name", sorted(GOLD["ib"]))
def test_oracle_ib_primitives_match_reference(oracle, name):
    g = GOLD["ib"][name]
    c = g["case"]
    kern = 1 if c["variant"] == "srt_peskin" else 0
    o = oracle.Oracle(c["nx"], c["ny"], tau0=c["tau"], u_in=0.1, delta_kernel=kern)
    o.step(c["pre_steps"], 1)
    for f, fid in (("ux", oracle.UX), ("uy", oracle.UY), ("rho", oracle.RHO)):
        assert sha(o.get(fid)) == g["pre_hash"][f]
    xy = np.array(g["xy"])
    o.set_markers(xy)
    vref, mf, nf = o.ib_probe(len(xy))
    assert vref.tolist() == g["vref"]
    assert mf.tolist() == g["mforce"]
    assert sha(nf) == g["nforce_hash"]
    assert sha(o.get(oracle.UX)) == g["ux_after_hash"]


def test_peskin_partition_of_unity(oracle):
    L = oracle.lib()
    for r0 in np.linspace(0.0, 1.0, 17):
        xs = [r0 + d for d in (-2, -1, 0, 1, 2)]
        phi = [L.orc_peskin_phi(x) for x in xs]
        assert abs(sum(phi) - 1.0) < 1e-14
        assert abs(sum(p * x for p, x in zip(phi, xs))) < 1e-14


def feq(rho, ux, uy):
    e = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]])
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    eu = e[:, 0] * ux + e[:, 1] * uy
    return w * rho * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * (ux * ux + uy * uy))


@pytest.mark.parametrize("coll", [0, 1, 2])
def test_equilibrium_is_fixed_point(oracle, coll):
    import ctypes as C

    L = oracle.lib()
    f = np.ascontiguousarray(feq(1.02, 0.05, -0.03))
    out = np.zeros(9)
    L.orc_collide_node(coll, f.ctypes.data_as(C.POINTER(C.c_double)), 1.02, 0.05, -0.03, 0.6,
                       out.ctypes.data_as(C.POINTER(C.c_double)))
    np.testing.assert_allclose(out, f, rtol=0, atol=1e-15)


def test_rr_tau_one_gives_equilibrium(oracle):
    import ctypes as C

    L = oracle.lib()
    rng = np.random.default_rng(3)
    f = np.ascontiguousarray(feq(1.0, 0.04, 0.01) + rng.uniform(-1e-3, 1e-3, 9))
    rho = f.sum()
    e = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]])
    ux, uy = (f * e[:, 0]).sum() / rho, (f * e[:, 1]).sum() / rho
    out = np.zeros(9)
    L.orc_collide_node(2, f.ctypes.data_as(C.POINTER(C.c_double)), rho, ux, uy, 1.0,
                       out.ctypes.data_as(C.POINTER(C.c_double)))
    np.testing.assert_allclose(out, feq(rho, ux, uy), rtol=0, atol=1e-15)


def test_channel_rest_state_stays_at_rest(oracle):
    o = oracle.Oracle(40, 20, bc_set=oracle.BC_CHANNEL, u_in=0.0, tau0=0.7)
    o.step(50, 1)
    assert np.abs(o.get(oracle.UX)).max() < 1e-15
    assert np.abs(o.get(oracle.RHO) - 1).max() < 1e-14


def test_channel_poiseuille_profile_is_steady(oracle):
    """Parabolic Zou-He inlet + zero-gradient outlet + halfway bounce-back
    walls: the Poiseuille profile u(y) = 4 u_max (y+1/2)(H-y-1/2)/H^2 is a
    steady state of the channel (to second order in the lattice)."""
    nx, ny, umax = 60, 24, 0.05
    y = np.arange(ny) + 0.5
    prof = 4 * umax * y * (ny - y) / ny ** 2
    ux = np.tile(prof[:, None], (1, nx))
    o = oracle.Oracle(nx, ny, bc_set=oracle.BC_CHANNEL, u_in=umax, tau0=0.8, les_model=0)
    o.init_macros(np.ones((ny, nx)), ux, np.zeros((ny, nx)))
    o.step(3000, 1)
    u = o.get(oracle.UX)
    err = np.abs(u[:, nx // 2] - prof).max() / umax
    assert err < 2e-2, err
    assert np.abs(o.get(oracle.UY)).max() < 1e-3 * umax * 10


def test_channel_cylinder_mass_and_force_sign(oracle):
    """A cylinder of IB markers in the channel feels a positive drag."""
    nx, ny = 120, 40
    n = 38
    th = 2 * np.pi * np.arange(n) / n
    xy = np.stack([30 + 6 * np.sin(th), 20 + 6 * np.cos(th)], axis=1)
    o = oracle.Oracle(nx, ny, bc_set=oracle.BC_CHANNEL, u_in=0.05, tau0=0.6, les_model=0,
                      delta_kernel=1)
    o.set_markers(xy, ds=np.full(n, 2 * np.pi * 6 / n))
    o.step(400, 1)
    (fx, fy), = o.forces()[0]
    assert fx > 0
    assert abs(fy) < 0.2 * fx


def test_mrt_and_bgk_agree_on_conserved_and_shear_moments(oracle):
    """The Lallemand-Luo MRT relaxes the two stress moments (p_xx - p_yy and
    p_xy) at s_nu = 1/tau, as BGK relaxes every moment: from the same
    post-stream populations both collisions give the same density, momentum
    and shear moments (the other moments relax at their own rates)."""
    import ctypes as C

    L = oracle.lib()
    rng = np.random.default_rng(11)
    e = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]], float)
    for tau in (0.52, 0.6, 0.9, 1.4):
        f = np.ascontiguousarray(feq(1.01, 0.03, -0.02) + rng.uniform(-2e-3, 2e-3, 9))
        rho = f.sum()
        ux, uy = (f * e[:, 0]).sum() / rho, (f * e[:, 1]).sum() / rho
        out = {}
        for coll in (0, 1):
            o = np.zeros(9)
            L.orc_collide_node(coll, f.ctypes.data_as(C.POINTER(C.c_double)), rho, ux, uy, tau,
                               o.ctypes.data_as(C.POINTER(C.c_double)))
            out[coll] = o
        for m in (np.ones(9), e[:, 0], e[:, 1], e[:, 0] ** 2 - e[:, 1] ** 2, e[:, 0] * e[:, 1]):
            assert (out[0] * m).sum() == pytest.approx((out[1] * m).sum(), abs=1e-15)
        # and the other moments do differ (the MRT is not BGK in disguise)
        q = e[:, 0] ** 2 + e[:, 1] ** 2
        assert abs((out[0] * q).sum() - (out[1] * q).sum()) > 1e-9


def test_oracle_runs_clean_under_address_and_undefined_behaviour_sanitizers(tmp_path):
    """The oracle's C code, built with -fsanitize=address,undefined, through
    its plate, channel, IB, solid and closure paths (tests/oracle_sanitize.c)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    here = os.path.dirname(os.path.abspath(__file__))
    odir = os.path.join(os.path.dirname(here), "oracle")
    exe = str(tmp_path / "oracle_sanitize")
    r = subprocess.run([gcc, "-std=gnu11", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
                        "-fno-sanitize-recover=undefined", "-I", odir, os.path.join(here, "oracle_sanitize.c"),
                        os.path.join(odir, "ippi_oracle.c"), "-lm", "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, ASAN_OPTIONS="detect_leaks=1"))
    assert r.returncode == 0 and "ok" in r.stdout, (r.stdout + r.stderr)[-3000:]


_THREAD_CHECK = r"""
import hashlib, sys
sys.path[:0] = sys.argv[1:3]
import pyoracle as po
from ippi_lbm import scenes
sc = scenes.cylinder_channel(256, 96, 24, 80, 48, 0.04, 3900)
p = dict(sc["params"]); p.pop("storage")
o = po.Oracle(256, 96, **p)
o.init_macros(*sc["init"])
o.set_markers(sc["markers"], ds=sc["ds"])
o.step(8, 1)
h = hashlib.sha256()
for f in (po.F, po.RHO, po.UX, po.UY, po.TAU):
    h.update(o.get(f).tobytes())
h.update(o.forces()[0].tobytes())
print(po.threads(), h.hexdigest())
"""


def test_threaded_loops_give_the_same_bytes(oracle):
    """The oracle's per-node loops run on OpenMP threads; every node's
    arithmetic is the same whatever the thread count, so an MRT +
    Smagorinsky channel with an IB cylinder gives identical bytes on 1 and 4
    threads."""
    import subprocess
    import sys

    from conftest import PKG_DIR, REPO

    out = {}
    for n in (1, 4):
        env = dict(os.environ, OMP_NUM_THREADS=str(n))
        r = subprocess.run([sys.executable, "-c", _THREAD_CHECK, os.path.join(REPO, "oracle"), PKG_DIR],
                           env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        threads, digest = r.stdout.split()
        assert int(threads) == n
        out[n] = digest
    assert out[1] == out[4]


def test_reference_on_libtorch_matches_the_stand_in_build(oracle, monkeypatch):
    """The reference compiled against libtorch (its boundary nets run by
    libtorch on the shipped TorchScript archives) and the stand-in build (the
    nets' forward restated in FP32) give the same plate with the nets on:
    populations and moments to FP32 rounding of the net output, identical
    net flags."""
    if not oracle.ref_available("srt_torch") or not oracle.ref_available("srt"):
        pytest.skip("reference builds absent (oracle/build_ref.sh)")
    monkeypatch.setenv("IPPI_REF_NN_DIR", os.path.join(GOLDEN, "band_nets"))
    a = oracle.RefSim(416, 12, tau=0.52, variant="srt_torch")
    b = oracle.RefSim(416, 12, tau=0.52, variant="srt")
    a.step(10, 1)
    b.step(10, 1)
    assert np.array_equal(a.get(oracle.NNFLAG), b.get(oracle.NNFLAG))
    assert a.get(oracle.NNFLAG).sum() > 0
    for f in (oracle.F, oracle.RHO, oracle.UX, oracle.UY):
        assert np.abs(a.get(f) - b.get(f)).max() < 1e-7
    assert np.abs(a.get(oracle.TAU) - b.get(oracle.TAU)).max() < 1e-6
