"""GPU checks of the learned relaxation time: the training kernels against
the FP64 restatement, the fused learned tau in the step against the FP64
oracle, the Smagorinsky fallback, the filtered-snapshot kernel, and a small
end-to-end run of the data -> training -> coarse-run pipeline."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
ip = pytest.importorskip("ippi_lbm")
import pyoracle as po  # noqa: E402
import tau_mlp as tm  # noqa: E402
from ippi_lbm import _lib  # noqa: E402
from ippi_lbm import learned_tau as lt  # noqa: E402
from ippi_lbm import scenes  # noqa: E402

DEV = torch.device("cuda", 0)


def dev(a, dtype=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV, dtype)


def stream():
    return torch.cuda.current_stream(DEV).cuda_stream


def gpu_grad(w, x, y):
    L = _lib.lib()
    wd, xd, yd = dev(w), dev(x), dev(y)
    g = torch.zeros(tm.NPARAM, dtype=torch.float32, device=DEV)
    loss = torch.zeros(1, dtype=torch.float32, device=DEV)
    scratch = torch.zeros(int(L.ippi_mlp_scratch_floats()), dtype=torch.float32, device=DEV)
    _lib.check(L.ippi_mlp_grad(xd.data_ptr(), yd.data_ptr(), x.shape[0], wd.data_ptr(), g.data_ptr(),
                               loss.data_ptr(), scratch.data_ptr(), stream()))
    torch.cuda.synchronize()
    return float(loss.item()), g.cpu().numpy().astype(np.float64)


def test_grad_kernel_matches_fp64_restatement_and_is_deterministic():
    rng = np.random.default_rng(0)
    w = (tm.xavier_init(1) + rng.normal(0, 0.05, tm.NPARAM)).astype(np.float32)
    x = rng.normal(0, 1, (5003, 6)).astype(np.float32)  # not a multiple of 32
    y = np.abs(rng.normal(0.8, 0.4, 5003)).astype(np.float32)
    loss, g = gpu_grad(w, x, y)
    lref, gref = tm.loss_and_grad(w.astype(np.float64), x.astype(np.float64), y.astype(np.float64))
    assert loss == pytest.approx(lref, rel=1e-5)
    assert np.abs(g - gref).max() <= 2e-5 * np.abs(gref).max()
    loss2, g2 = gpu_grad(w, x, y)
    assert loss2 == loss and np.array_equal(g, g2)


def test_forward_and_adam_kernels():
    L = _lib.lib()
    rng = np.random.default_rng(1)
    w = (tm.xavier_init(2) + rng.normal(0, 0.05, tm.NPARAM)).astype(np.float32)
    x = rng.normal(0, 1, (777, 6)).astype(np.float32)
    out = torch.empty(777, dtype=torch.float32, device=DEV)
    wd, xd = dev(w), dev(x)
    _lib.check(L.ippi_mlp_forward(xd.data_ptr(), 777, wd.data_ptr(), out.data_ptr(), stream()))
    ref = tm.forward(w.astype(np.float64), x.astype(np.float64))
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=2e-6, atol=1e-7)
    # three Adam steps
    g = rng.normal(0, 1e-2, tm.NPARAM)
    m = np.zeros(tm.NPARAM)
    v = np.zeros(tm.NPARAM)
    wr = w.astype(np.float64).copy()
    md, vd, gd = dev(m), dev(v), dev(g)
    for step in (1, 2, 3):
        tm.adam(wr, g, m, v, step, 1e-3)
        _lib.check(L.ippi_mlp_adam(wd.data_ptr(), gd.data_ptr(), md.data_ptr(), vd.data_ptr(), step,
                                   1e-3, 0.9, 0.999, 1e-8, stream()))
    np.testing.assert_allclose(wd.cpu().numpy(), wr, rtol=0, atol=2e-6)


def test_training_fits_a_teacher_network():
    rng = np.random.default_rng(4)
    teacher = tm.xavier_init(11) * 1.5
    x = rng.normal(0, 1, (65536, 6))
    y = tm.forward(teacher, x)
    net, hist = lt.train(x, y, epochs=30, batch=4096, lr=3e-3, seed=0, clip_pct=100)
    assert hist[-1] < 0.05 * hist[0], hist
    pred = lt.predict(net, x[:4096], bf16=False)
    assert np.sqrt(np.mean((pred - y[:4096]) ** 2)) < 0.1 * np.std(y)


def _learned_pair(storage, coll, nx=160, ny=48, lo_all=None):
    kw = dict(collision=coll, bc_set=ip.BC_CHANNEL, tau0=0.505, cs=0.1, u_in=0.05,
              delta_kernel=ip.DELTA_PESKIN4, les_model=ip.LES_LEARNED)
    o = po.Oracle(nx, ny, **kw)
    g = ip.Lattice(nx, ny, storage=storage, **kw)
    rng = np.random.default_rng(5)
    w = tm.xavier_init(5) + rng.normal(0, 0.1, tm.NPARAM)
    bits, wv = lt.bf16_bits(w)
    mean = np.array([1.0, 0.04, 0.0, 0.0, 0.0, 2e-3])
    std = np.array([1e-3, 0.02, 0.5, 0.5, 0.5, 2e-3])
    lo = np.array([0.95, 0.0, -1.0, -1.0, -1.0, 0.0]) if lo_all is None else np.full(6, lo_all)
    hi = np.array([1.05, 0.2, 1.0, 1.0, 1.0, 0.05]) if lo_all is None else np.full(6, 2 * lo_all)
    stats = np.concatenate([mean, std, lo, hi, [0.01]]).astype(np.float32)
    o.load_tau_mlp(wv, stats)
    g.load_tau_mlp(bits, stats)
    sc = scenes.cylinder_channel(nx, ny, 12, 40.3, 24.1, 0.05, 100, collision=coll)
    o.set_markers(sc["markers"], ds=sc["ds"])
    g.set_markers(sc["markers"], ds=sc["ds"])
    o.init_macros(*sc["init"])
    g.init_macros(*sc["init"])
    return o, g


@pytest.mark.parametrize("coll", [ip.MRT, ip.BGK, ip.RR])
def test_fused_learned_tau_fp64_matches_oracle(coll):
    o, g = _learned_pair(ip.F64, coll)
    for n, t0 in ((1, 1), (19, 2)):
        o.step(n, t0)
        g.step(n, t0)
        tau_o, tau_g = o.get(po.TAU), g.download(ip.FIELD_TAU)
        assert np.abs(tau_g - tau_o).max() < 1e-12
        assert np.abs(tau_o - 0.505).max() > 1e-3  # the network changes tau
        f_o, f_g = o.get(po.F), g.download(ip.FIELD_F)
        assert np.abs(f_g - f_o).max() / np.abs(f_o).max() < 1e-11
        np.testing.assert_allclose(g.forces(), o.forces()[0], rtol=1e-9, atol=1e-13)


def test_fused_learned_tau_fp32_tolerance():
    o, g = _learned_pair(ip.F32, ip.MRT)
    o.step(1, 1)
    g.step(1, 1)
    assert np.abs(g.download(ip.FIELD_TAU) - o.get(po.TAU)).max() < 1e-5
    o.step(30, 2)
    g.step(30, 2)
    f_o = o.get(po.F)
    assert np.abs(g.download(ip.FIELD_F) - f_o).max() / np.abs(f_o).max() < 2e-4


def test_out_of_range_features_fall_back_to_smagorinsky():
    # a training range no node reaches: every node takes the Smagorinsky tau
    _, g = _learned_pair(ip.F64, ip.MRT, lo_all=1e6)
    sc = scenes.cylinder_channel(160, 48, 12, 40.3, 24.1, 0.05, 100, collision=ip.MRT)
    r = ip.Lattice(160, 48, storage=ip.F64, collision=ip.MRT, bc_set=ip.BC_CHANNEL, tau0=0.505,
                   cs=0.1, u_in=0.05, delta_kernel=ip.DELTA_PESKIN4, les_model=ip.LES_SMAGORINSKY)
    r.set_markers(sc["markers"], ds=sc["ds"])
    r.init_macros(*sc["init"])
    g.step(10, 1)
    r.step(10, 1)
    assert np.abs(g.download(ip.FIELD_TAU) - r.download(ip.FIELD_TAU)).max() < 1e-14
    assert np.abs(g.download(ip.FIELD_F) - r.download(ip.FIELD_F)).max() < 1e-13


def test_learned_tau_needs_a_network_and_the_channel_scene():
    g = ip.Lattice(64, 32, bc_set=ip.BC_CHANNEL, u_in=0.05, tau0=0.6, les_model=ip.LES_LEARNED)
    with pytest.raises(ip.IppiError, match="no network"):
        g.step(1, 1)
    with pytest.raises(ip.IppiError):
        ip.Lattice(64, 32, les_model=ip.LES_LEARNED)  # flat plate
    with pytest.raises(ip.IppiError):
        g.load_tau_mlp(np.zeros(10, np.uint16), np.ones(25, np.float32))


def test_filter_snapshot_matches_host_box_filter():
    nx, ny, fac = 96, 48, 4
    sc = scenes.cylinder_channel(nx, ny, 12, 30.3, 24.1, 0.05, 100, collision=ip.MRT,
                                 storage=ip.F64)
    g = ip.Lattice(nx, ny, **sc["params"])
    g.init_macros(*sc["init"])
    g.set_markers(sc["markers"], ds=sc["ds"])
    g.step(25, 1)
    snap = g.filter_snapshot(fac)
    f = g.download(ip.FIELD_F)
    rho, ux, uy = (g.download(k) for k in (ip.FIELD_RHO, ip.FIELD_UX, ip.FIELD_UY))
    tau = g.download(ip.FIELD_TAU)
    d = f[5] + f[6] + f[7] + f[8]
    pxx = f[1] + f[3] + d - rho / 3 - rho * ux * ux
    pyy = f[2] + f[4] + d - rho / 3 - rho * uy * uy
    pxy = f[5] - f[6] + f[7] - f[8] - rho * ux * uy
    c = -(1 - 0.5 / tau)

    def box(a):
        return a.reshape(ny // fac, fac, nx // fac, fac).mean(axis=(1, 3))

    rb = box(rho)
    ub, vb = box(rho * ux) / rb, box(rho * uy) / rb
    want = [rb, ub, vb, box(c * pxx) - (box(rho * ux * ux) - rb * ub * ub),
            box(c * pxy) - (box(rho * ux * uy) - rb * ub * vb),
            box(c * pyy) - (box(rho * uy * uy) - rb * vb * vb)]
    for k in range(6):
        scale = max(np.abs(want[k]).max(), 1e-30)
        assert np.abs(snap[k] - want[k]).max() / scale < 1e-10, k


def test_pipeline_small_end_to_end():
    """Fine 512 x 128 (D = 32) -> filtered x4 -> train -> coarse 128 x 32
    learned run: stable, finite forces, network beats Smagorinsky on the
    held-out targets."""
    fine = scenes.cylinder_channel(512, 128, 32, 128, 64, 0.05, 300, collision=ip.MRT)
    res = lt.run_cylinder(fine, 3000, 2001, snapshot=(4, 2000, 50, 20))
    snaps = res["snapshots"]
    assert len(snaps) == 20
    tau0c = 3 * 0.05 * 8 / 300 + 0.5
    mask = lt.cylinder_mask(128, 32, 32, 16, 8)
    xs, ys = zip(*(lt.samples_from_snapshot(s, tau0c, mask) for s in snaps))
    xtr, ytr = np.concatenate(xs[:16]), np.concatenate(ys[:16])
    xte, yte = np.concatenate(xs[16:]), np.concatenate(ys[16:])
    net, hist = lt.train(xtr, ytr, epochs=20, batch=1024, lr=3e-3)
    assert hist[-1] < hist[0]
    pred = lt.predict(net, xte)
    # Smagorinsky tau on the same features (|S| there is the tau0-based estimate)
    q = xte[:, 5]
    smag = 0.5 * (np.sqrt(tau0c ** 2 + 18 * 0.1 ** 2 * q / xte[:, 0]) + tau0c) - tau0c
    yclip = np.minimum(yte, np.percentile(ytr, 99.5))
    assert np.mean((pred - yclip) ** 2) < np.mean((smag - yclip) ** 2)
    coarse = scenes.cylinder_channel(128, 32, 8, 32, 16, 0.05, 300, collision=ip.MRT)
    out = lt.run_cylinder(coarse, 1500, 1001, net=net)
    assert np.isfinite(out["cd"]) and out["cd"] > 0


def test_experiment_driver_small():
    """The learned-tau experiment driver end to end on a small channel (the
    code path behind the bench's learned mode): fine run, filtered snapshots,
    a-priori training, training through the solver on the filtered field,
    the wake-velocity scale fit, the coarse runs and the plain resolution
    ladder, with every reported figure finite."""
    r = lt.experiment(nx=512, ny=128, d=32, u=0.05, re=300.0, fine_steps=2000, avg_steps=800,
                      n_snap=10, epochs=3, fine_seeds=(0, 1), eval_seeds=(0, 1), field_iters=2,
                      wake_grid=(1, 4), wake_iters=2, ladder=(16,))
    for k in ("plain", "a_priori", "through_solver_field", "a_priori_wake_scale"):
        assert np.isfinite(r[k]["cd"]) and r[k]["cd"] > 0, k
        assert r[k]["wall_s"] > 0 and len(r[k]["cd_per_seed"]) == 2, k
    assert np.isfinite(r["fine"]["cd"]) and r["fine"]["cd_seed_spread"] is not None
    assert r["coarse"]["nx"] == 128 and r["coarse"]["steps"] == 500
    assert r["field_training"]["iters"] == 2 and r["field_training"]["horizon"] == 20
    assert r["wake_fit"]["runs"] == 4 and r["ladder"][0]["nx"] == 256
    assert set(r["time_to_solution"]) == {"a_priori", "through_solver_field", "a_priori_wake_scale"}
    assert r["training"]["samples"] > 0


def _learned_lattice(seed, storage=ip.F32):
    kw = dict(collision=ip.MRT, bc_set=ip.BC_CHANNEL, tau0=0.505, cs=0.1, u_in=0.05,
              delta_kernel=ip.DELTA_PESKIN4, les_model=ip.LES_LEARNED, storage=storage)
    g = ip.Lattice(160, 48, **kw)
    rng = np.random.default_rng(seed)
    bits, _ = lt.bf16_bits(tm.xavier_init(seed) + rng.normal(0, 0.1, tm.NPARAM))
    stats = np.concatenate([[1.0, 0.04, 0, 0, 0, 2e-3], [1e-3, 0.02, 0.5, 0.5, 0.5, 2e-3],
                            [-1e6] * 6, [1e6] * 6, [0.01]]).astype(np.float32)
    g.load_tau_mlp(bits, stats)
    sc = scenes.cylinder_channel(160, 48, 12, 40.3, 24.1, 0.05, 100, collision=ip.MRT)
    g.set_markers(sc["markers"], ds=sc["ds"])
    g.init_macros(*sc["init"])
    return g


def test_networks_of_several_handles_take_turns_in_constant_memory():
    """The fused kernels read the network from constant memory, one network
    per device at a time: handles with different networks, stepped and read
    in alternation or from two host threads at once, give exactly what each
    gives alone."""
    import threading

    solo = {}
    for seed in (1, 2):
        g = _learned_lattice(seed)
        g.step(20, 1)
        solo[seed] = (g.download(ip.FIELD_F), g.download(ip.FIELD_TAU))
        g.close()
    assert not np.array_equal(solo[1][1], solo[2][1])
    a = {s: _learned_lattice(s) for s in (1, 2)}
    for k in range(4):
        for s in (1, 2):
            a[s].step(5, 1 + 5 * k)
    for s in (2, 1):  # downloads re-run the last step with the handle's network
        assert np.array_equal(a[s].download(ip.FIELD_TAU), solo[s][1])
        assert np.array_equal(a[s].download(ip.FIELD_F), solo[s][0])
    b = {s: _learned_lattice(s) for s in (1, 2)}
    errs = []

    def run(s):
        try:
            for t in range(1, 21):
                b[s].step(1, t)
        except Exception as e:  # reported below
            errs.append(e)

    th = [threading.Thread(target=run, args=(s,)) for s in (1, 2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs
    for s in (1, 2):
        assert np.array_equal(b[s].download(ip.FIELD_F), solo[s][0])


def _tc_pair(storage=ip.F32):
    """Two learned lattices from the same seeded network (range covering every
    node): the hidden layer on FMA and on the tensor cores."""
    out = []
    for tc in (False, True):
        g = _learned_lattice(2, storage)
        if tc:
            g.set_learned_tensor_cores(True)
        out.append(g)
    return out


def test_tensor_core_network_matches_the_fma_network():
    """The learned tau's 32 x 32 hidden layer on the tensor cores (BF16
    activations and weights, FP32 accumulation, mma.sync m16n8k16 over the
    32 nodes of a warp) against the FMA network: after 1 step the
    populations agree to 1e-6 of max |f|, after 40 steps to 1e-4; the body
    forces to 1e-3.  The network has not gone missing: switching it off
    again gives the FMA lattice's bits."""
    a, b = _tc_pair()
    for n, t0, tol in ((1, 1, 1e-6), (39, 2, 1e-4)):
        a.step(n, t0)
        b.step(n, t0)
        fa, fb = a.download(ip.FIELD_F), b.download(ip.FIELD_F)
        assert np.abs(fa - fb).max() <= tol * np.abs(fa).max(), (n, np.abs(fa - fb).max())
    assert np.abs(fa - fb).max() > 0  # BF16 activations do change the result
    np.testing.assert_allclose(b.forces(), a.forces(), rtol=1e-3, atol=1e-6)
    c, d = _learned_lattice(3), _learned_lattice(3)
    d.set_learned_tensor_cores(True)
    d.set_learned_tensor_cores(False)
    c.step(10, 1)
    d.step(10, 1)
    assert np.array_equal(c.download(ip.FIELD_F), d.download(ip.FIELD_F))


def test_tensor_core_network_is_refused_where_it_does_not_apply():
    g = _learned_lattice(1, ip.F64)
    with pytest.raises(ip.IppiError, match="FP32 arithmetic"):
        g.set_learned_tensor_cores(True)
    plain = ip.Lattice(64, 32, collision=ip.MRT, bc_set=ip.BC_CHANNEL, u_in=0.05, tau0=0.56,
                       storage=ip.F32)
    with pytest.raises(ip.IppiError, match="IPPI_LES_LEARNED"):
        plain.set_learned_tensor_cores(True)
    h = _learned_lattice(1)
    h.set_learned_tensor_cores(True)
    h.step(2, 1)
    with pytest.raises(ip.IppiError, match="tensor cores off"):
        h.adjoint_forward(4, 3, 2)
