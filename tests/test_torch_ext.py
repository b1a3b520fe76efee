"""The libtorch extension (torch_ext/ippi_autograd.cpp): torch::autograd::Function
wrappers of a rollout whose forward is the checkpointed GPU rollout and whose
backward is the library's adjoint.

CPU: the in-tree extension loads, exposes its two rollout factories, and
rejects a null lattice handle.  GPU: on the same lattice, loss weights and
parameters, the C++ Function's loss and gradient equal the Python
torch.autograd.Function's and the direct ippi_adjoint_backward call's, for
the tau field and for the network weights; a second forward/backward of the
same rollout (state restored from the captured checkpoint) gives the same
bits.
"""
import numpy as np
import pytest

ip = pytest.importorskip("ippi_lbm")
torch = pytest.importorskip("torch")
from ippi_lbm import autograd as ag  # noqa: E402


def test_extension_loads_and_checks_its_handle():
    ext = ag.native()
    assert hasattr(ext, "tau_field_rollout") and hasattr(ext, "network_rollout")
    with pytest.raises(RuntimeError, match="null lattice handle"):
        ext.tau_field_rollout(0, 10, 1, 4, torch.zeros(4, 4, dtype=torch.float64))


@pytest.mark.gpu
def test_tau_field_function_matches_python_wrapper_and_adjoint():
    import tau_mlp  # noqa: F401  (oracle path on sys.path via conftest)
    from test_adjoint_gpu import PRE, loss_weights, run_gpu, setup, smooth_field

    nx, ny, nsteps = 64, 32, 20
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_FIELD, seed=3)
    tau0 = 0.56 + smooth_field(rng, ny, nx, 0.02)
    tau1 = tau0 + smooth_field(rng, ny, nx, 0.005)
    a, b = loss_weights(rng, nsteps, nx, ny)
    lat = ip.Lattice(nx, ny, **p)
    lat.set_markers(sc["markers"], ds=sc["ds"])
    lat.init_macros(*sc["init"])
    lat.set_tau_field(tau0)
    lat.step(PRE, 1)
    roll = ag.native().tau_field_rollout(lat.handle.value, nsteps, PRE + 1, 7, torch.from_numpy(tau0))
    grads, losses = [], []
    for _ in range(2):
        tau = torch.tensor(tau1, dtype=torch.float64, requires_grad=True)
        forces, macros = roll(tau)
        loss = (forces * torch.from_numpy(a)).sum() + (macros * torch.from_numpy(b)).sum()
        loss.backward()
        grads.append(tau.grad.numpy().copy())
        losses.append(float(loss.detach()))
    assert np.array_equal(grads[0], grads[1]) and losses[0] == losses[1]
    # the direct adjoint call from the same starting state
    L0, g = run_gpu(sc, p, nsteps, a, b, tau=tau1, base=tau0, grads=dict(tau=True))
    assert losses[0] == pytest.approx(L0, rel=1e-12)
    np.testing.assert_allclose(grads[0], g["tau"], rtol=1e-10, atol=1e-14)
    # the Python torch.autograd.Function
    lat2 = ip.Lattice(nx, ny, **p)
    lat2.set_markers(sc["markers"], ds=sc["ds"])

    def reset(lt_):
        lt_.init_macros(*sc["init"])
        lt_.set_tau_field(tau0)
        lt_.step(PRE, 1)

    tau = torch.tensor(tau1, dtype=torch.float64, requires_grad=True)
    forces, macros = ag.TauFieldRollout.apply(tau, ag.Rollout(lat2, reset, nsteps, PRE + 1, 7))
    ((forces * torch.from_numpy(a)).sum() + (macros * torch.from_numpy(b)).sum()).backward()
    np.testing.assert_allclose(grads[0], tau.grad.numpy(), rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_network_function_matches_adjoint():
    import tau_mlp as tm
    from test_adjoint_gpu import PRE, loss_weights, run_gpu, setup

    nx, ny, nsteps = 64, 32, 20
    sc, p, rng = setup(nx, ny, ip.MRT, ip.LES_LEARNED, seed=6)
    w0 = (tm.xavier_init(3) + rng.normal(0, 0.1, tm.NPARAM)).astype(np.float32)
    w1 = (w0 + rng.normal(0, 0.01, tm.NPARAM)).astype(np.float32)
    stats = np.concatenate([[1.0, 0.03, 0, 0, 0, 5e-3], [2e-3, 0.02, 0.5, 0.5, 0.5, 5e-3],
                            [0.9, 0.0, -1, -1, -1, 0.0], [1.1, 0.2, 1, 1, 1, 0.2],
                            [0.02]]).astype(np.float32)
    a, b = loss_weights(rng, nsteps, nx, ny)
    lat = ip.Lattice(nx, ny, **p)
    lat.set_markers(sc["markers"], ds=sc["ds"])
    lat.init_macros(*sc["init"])
    lat.load_tau_mlp_f32(w0, stats)
    lat.step(PRE, 1)
    roll = ag.native().network_rollout(lat.handle.value, nx, ny, nsteps, PRE + 1, 7, torch.from_numpy(w0),
                                       torch.from_numpy(stats))
    w = torch.tensor(w1, requires_grad=True)
    forces, macros = roll(w)
    loss = (forces * torch.from_numpy(a)).sum() + (macros * torch.from_numpy(b)).sum()
    loss.backward()
    assert w.grad.dtype == torch.float32
    L0, g = run_gpu(sc, p, nsteps, a, b, w=w1, stats=stats, base=w0, grads=dict(mlp=True))
    assert float(loss.detach()) == pytest.approx(L0, rel=1e-12)
    np.testing.assert_allclose(w.grad.numpy(), g["mlp"].astype(np.float32), rtol=1e-6, atol=1e-12)
