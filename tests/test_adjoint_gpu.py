"""Reverse-mode gradients through the step (ippi_adjoint_forward / _backward)
against central finite differences of the FP64 forward: on the GPU itself and
on the FP64 CPU oracle.  The loss mixes every output the adjoint accepts: a
weighted sum of the per-step body forces and of the final post-stream rho,
ux, uy.  Every run first advances PRE steps with the unperturbed parameters,
so the state the rollout starts from is the same for all of them (the
gradient is taken with that state held fixed)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402
import tau_mlp as tm  # noqa: E402
from ippi_lbm import scenes  # noqa: E402


def setup(nx, ny, coll, les, seed=0):
    sc = scenes.cylinder_channel(nx, ny, 8, 16.3, ny / 2 + 0.1, 0.05, 60, collision=coll,
                                 storage=ip.F64)
    p = dict(sc["params"])
    p.update(les_model=les, tau0=0.56, cs=0.1)
    rng = np.random.default_rng(seed)
    return sc, p, rng


def loss_weights(rng, nsteps, nx, ny):
    a = rng.normal(0, 1, (nsteps, 1, 2))
    b = rng.normal(0, 1e-2, (3, ny, nx))
    return a, b


PRE = 3


def run_gpu(sc, p, nsteps, a, b, tau=None, w=None, stats=None, K=7, grads=None, base=None):
    g = ip.Lattice(sc["nx"], sc["ny"], **p)
    g.init_macros(*sc["init"])
    g.set_markers(sc["markers"], ds=sc["ds"])
    if tau is not None:
        g.set_tau_field(base if base is not None else tau)
    if w is not None:
        g.load_tau_mlp_f32(base if base is not None else w, stats)
    g.step(PRE, 1)
    if tau is not None:
        g.set_tau_field(tau)
    if w is not None:
        g.load_tau_mlp_f32(w, stats)
    g.adjoint_forward(nsteps, PRE + 1, K)
    F = g.force_history(nsteps)
    m = np.stack([g.download(k) for k in (ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY)])
    L = float(np.sum(a * F) + np.sum(b * m))
    out = None
    if grads:
        out = g.adjoint_backward(dl_dforce=a, dl_dmacro=b, **grads)
    g.close()
    return L, out


def smooth_field(rng, ny, nx, amp):
    yy, xx = np.mgrid[0:ny, 0:nx]
    f = np.zeros((ny, nx))
    for _ in range(4):
        kx, ky = rng.uniform(0.05, 0.3, 2)
        f += np.sin(kx * xx + rng.uniform(0, 6)) * np.cos(ky * yy + rng.uniform(0, 6))
    return amp * f / 4


@pytest.mark.parametrize("coll", [ip.MRT, ip.BGK, ip.RR])
def test_tau_field_gradient_matches_finite_differences(coll):
    nx, ny, nsteps = 64, 32, 40
    sc, p, rng = setup(nx, ny, coll, ip.LES_FIELD)
    tau = 0.56 + smooth_field(rng, ny, nx, 0.03)
    a, b = loss_weights(rng, nsteps, nx, ny)
    L0, g = run_gpu(sc, p, nsteps, a, b, tau=tau, grads=dict(tau=True))
    grad = g["tau"]
    assert np.abs(grad).max() > 0
    eps = 1e-6
    for _ in range(5):
        d = rng.normal(0, 1, (ny, nx))
        lp, _ = run_gpu(sc, p, nsteps, a, b, tau=tau + eps * d, base=tau)
        lm, _ = run_gpu(sc, p, nsteps, a, b, tau=tau - eps * d, base=tau)
        fd = (lp - lm) / (2 * eps)
        ad = float(np.sum(grad * d))
        assert abs(fd - ad) <= 1e-5 * max(abs(fd), 1e-8), (fd, ad)


def test_network_weight_gradient_matches_finite_differences():
    nx, ny, nsteps = 64, 32, 30
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_LEARNED)
    w = (tm.xavier_init(3) + rng.normal(0, 0.1, tm.NPARAM)).astype(np.float32)
    stats = np.concatenate([[1.0, 0.03, 0, 0, 0, 5e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 5e-3],
                            [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.2],
                            [0.02]]).astype(np.float32)
    a, b = loss_weights(rng, nsteps, nx, ny)
    _, g = run_gpu(sc, p, nsteps, a, b, w=w, stats=stats, grads=dict(mlp=True))
    grad = g["mlp"]
    assert np.abs(grad).max() > 0
    # central differences with eps = 1e-3 and 5e-4, Richardson-combined (the
    # O(eps^2) truncation of a single difference is ~5e-4 relative here)
    for _ in range(5):
        d = rng.normal(0, 1, tm.NPARAM)
        dl, ad = [], []
        for eps in (1e-3, 5e-4):
            wp = (w + eps * d).astype(np.float32)
            wm = (w - eps * d).astype(np.float32)
            lp, _ = run_gpu(sc, p, nsteps, a, b, w=wp, stats=stats, base=w)
            lm, _ = run_gpu(sc, p, nsteps, a, b, w=wm, stats=stats, base=w)
            dl.append(lp - lm)
            # the exact float perturbation, so rounding of w +- eps d does not enter
            ad.append(float(grad @ (wp.astype(np.float64) - wm.astype(np.float64))))
        # dL(eps) = g.dw + c eps^3 + ...: 8 dL(eps/2) - dL(eps) cancels the cubic term
        fd = 8 * dl[1] - dl[0]
        want = 8 * ad[1] - ad[0]
        assert abs(fd - want) <= 2e-5 * max(abs(fd), 1e-12), (fd, want)


def test_backward_sweep_is_bit_reproducible():
    """The transposed streaming is a gather (each dL/df_in entry written once,
    no atomics) and every other reduction has a fixed order: two backward
    sweeps of the same rollout give the same bits, for the tau field and the
    network weights, on a channel whose outlet and inlet columns carry
    adjoint."""
    nx, ny, nsteps = 64, 32, 25
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_LEARNED, seed=4)
    w = (tm.xavier_init(7) + rng.normal(0, 0.1, tm.NPARAM)).astype(np.float32)
    stats = np.concatenate([[1.0, 0.03, 0, 0, 0, 5e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 5e-3],
                            [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.2],
                            [0.02]]).astype(np.float32)
    a, b = loss_weights(rng, nsteps, nx, ny)
    runs = [run_gpu(sc, p, nsteps, a, b, w=w, stats=stats, grads=dict(mlp=True, f0=True))[1] for _ in range(2)]
    assert np.abs(runs[0]["mlp"]).max() > 0
    for k in ("mlp", "f0"):
        assert np.array_equal(runs[0][k], runs[1][k]), k
    # the edge columns carry adjoint (the inlet's and outlet's transposes ran)
    f0 = runs[0]["f0"].reshape(9, ny, nx)
    assert np.abs(f0[:, :, 0]).max() > 0 and np.abs(f0[:, :, nx - 2]).max() > 0
    sc, p, rng = setup(nx, ny, ip.RR, ip.LES_FIELD, seed=5)
    tau = 0.56 + smooth_field(rng, ny, nx, 0.01)
    runs = [run_gpu(sc, p, nsteps, a, b, tau=tau, grads=dict(tau=True))[1]["tau"] for _ in range(2)]
    assert np.abs(runs[0]).max() > 0 and np.array_equal(runs[0], runs[1])


def test_gradient_matches_fp64_oracle_on_128x64_200_steps():
    """The adjoint's directional derivatives against central differences of
    the FP64 CPU oracle (an independent forward implementation)."""
    nx, ny, nsteps = 128, 64, 200
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_FIELD, seed=7)
    tau = 0.56 + smooth_field(rng, ny, nx, 0.03)
    a, b = loss_weights(rng, nsteps, nx, ny)
    _, g = run_gpu(sc, p, nsteps, a, b, tau=tau, K=64, grads=dict(tau=True))

    def oracle_loss(t):
        o = po.Oracle(nx, ny, collision=p["collision"], bc_set=po.BC_CHANNEL, les_model=3,
                      tau0=p["tau0"], cs=p["cs"], u_in=p["u_in"], delta_kernel=p["delta_kernel"],
                      mdf_iters=1)
        o.set_tau_field(tau)
        o.set_markers(sc["markers"], ds=sc["ds"])
        o.init_macros(*sc["init"])
        # An oracle step is IB + collision, then streaming: its step k holds the
        # collision the GPU performs at the end of its step k - 1.  The GPU
        # rollout's perturbed collisions are those of its steps PRE+1 ..;
        # here they sit in oracle steps PRE+2 ..; forces are tau-independent.
        assert o.step(PRE + 1, 1) == 0
        o.set_tau_field(t)
        F = np.zeros((nsteps, 1, 2))
        for s in range(nsteps):
            if s:
                assert o.step(1, PRE + s + 1) == 0
            F[s, 0] = o.forces()[0][:2]
        m = np.stack([o.get(k) for k in (po.RHO, po.UX, po.UY)])
        return float(np.sum(a * F) + np.sum(b * m))

    eps = 1e-6
    for _ in range(3):
        d = rng.normal(0, 1, (ny, nx))
        fd = (oracle_loss(tau + eps * d) - oracle_loss(tau - eps * d)) / (2 * eps)
        ad = float(np.sum(g["tau"] * d))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-8), (fd, ad)


def test_adjoint_argument_checks():
    g = ip.Lattice(64, 32)  # flat plate
    with pytest.raises(ip.IppiError):
        g.adjoint_forward(10)
    sc, p, _ = setup(64, 32, ip.MRT, ip.LES_SMAGORINSKY)
    g = ip.Lattice(64, 32, **p)
    with pytest.raises(ip.IppiError):
        g.adjoint_backward(tau=True)  # nothing recorded
    g.adjoint_forward(5, 1, 2)
    with pytest.raises(ip.IppiError, match="tau-field"):
        g.adjoint_backward(tau=True)


def test_torch_autograd_wrapper_gives_the_adjoint_gradient():
    torch = pytest.importorskip("torch")
    from ippi_lbm.autograd import Rollout, TauFieldRollout

    nx, ny, nsteps = 64, 32, 20
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_FIELD, seed=3)
    tau0 = 0.56 + smooth_field(rng, ny, nx, 0.02)
    a, b = loss_weights(rng, nsteps, nx, ny)
    lat = ip.Lattice(nx, ny, **p)
    lat.set_markers(sc["markers"], ds=sc["ds"])

    def reset(lt_):
        lt_.init_macros(*sc["init"])
        lt_.set_tau_field(tau0)
        lt_.step(PRE, 1)

    roll = Rollout(lat, reset, nsteps, PRE + 1, 7)
    tau = torch.tensor(tau0, dtype=torch.float64, requires_grad=True)
    forces, macros = TauFieldRollout.apply(tau, roll)
    loss = (forces * torch.from_numpy(a)).sum() + (macros * torch.from_numpy(b)).sum()
    loss.backward()
    L0, g = run_gpu(sc, p, nsteps, a, b, tau=tau0, grads=dict(tau=True))
    assert float(loss.detach()) == pytest.approx(L0, rel=1e-12)
    np.testing.assert_allclose(tau.grad.numpy(), g["tau"], rtol=1e-10, atol=1e-14)


ADJ_CHILD = """
import sys
sys.path[:0] = [%r, %r]
import numpy as np
import ippi_lbm as ip
import tau_mlp as tm
from ippi_lbm import scenes
out = []
for les in (ip.LES_FIELD, ip.LES_LEARNED, ip.LES_SMAGORINSKY):
    sc = scenes.cylinder_channel(64, 32, 8, 16.3, 16.1, 0.05, 60, collision=ip.MRT, storage=ip.F64)
    p = dict(sc["params"]); p.update(les_model=les, tau0=0.56, cs=0.1)
    g = ip.Lattice(64, 32, **p)
    g.init_macros(*sc["init"]); g.set_markers(sc["markers"], ds=sc["ds"])
    rng = np.random.default_rng(1)
    if les == ip.LES_FIELD:
        g.set_tau_field(0.56 + 0.02 * rng.random((32, 64)))
    if les == ip.LES_LEARNED:
        w = (tm.xavier_init(3) + rng.normal(0, 0.1, tm.NPARAM)).astype(np.float32)
        st = np.concatenate([[1.0, 0.03, 0, 0, 0, 5e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 5e-3],
                             [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.2], [0.02]]).astype(np.float32)
        g.load_tau_mlp_f32(w, st)
    g.step(3, 1)
    g.adjoint_forward(20, 4, 7)
    a = rng.normal(0, 1, (20, 1, 2)); b = rng.normal(0, 1e-2, (3, 32, 64))
    r = g.adjoint_backward(dl_dforce=a, dl_dmacro=b, tau=les == ip.LES_FIELD, mlp=les == ip.LES_LEARNED,
                           f0=True)
    out.append({k: np.asarray(v) for k, v in r.items() if v is not None})
    g.close()
np.savez(sys.argv[1], **{f"{i}_{k}": v for i, d in enumerate(out) for k, v in d.items()})
"""


def test_reverse_mode_mrt_collision_equals_dual_numbers(tmp_path):
    """The hand-written reverse-mode MRT collision adjoint against the dual-
    number kernel (IPPI_TEST_ADJ_DUAL=1) on the same rollouts: tau-field,
    network-weight and initial-population gradients, learned / field /
    Smagorinsky relaxation times, with IB markers."""
    import os
    import subprocess
    import sys

    from conftest import PKG_DIR, REPO

    code = ADJ_CHILD % (PKG_DIR, os.path.join(REPO, "oracle"))
    res = {}
    for mode in ("0", "1"):
        path = str(tmp_path / f"g{mode}.npz")
        env = dict(os.environ, IPPI_TEST_ADJ_DUAL=mode)
        r = subprocess.run([sys.executable, "-c", code, path], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        res[mode] = dict(np.load(path))
    assert res["0"].keys() == res["1"].keys() and len(res["0"]) >= 4
    for k in res["0"]:
        a, b = res["0"][k], res["1"][k]
        assert np.abs(b).max() > 0, k
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-10 * np.abs(b).max(), err_msg=k)
