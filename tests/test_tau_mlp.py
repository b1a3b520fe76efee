"""CPU checks of the learned relaxation time: the FP64 restatement
(oracle/tau_mlp.py) against finite differences, the C oracle's fused
learned_tau against it, BF16 rounding, and the training-target construction
on flows with known answers."""
import numpy as np
import pytest

import tau_mlp as tm
from ippi_lbm import learned_tau as lt


def test_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    w = tm.xavier_init(3) + rng.normal(0, 0.05, tm.NPARAM)
    x = rng.normal(0, 1, (37, 6))
    y = np.abs(rng.normal(0.5, 0.3, 37))
    loss, g = tm.loss_and_grad(w, x, y)
    for _ in range(20):
        d = rng.normal(0, 1, tm.NPARAM)
        d /= np.linalg.norm(d)
        eps = 1e-5
        fd = (tm.loss_and_grad(w + eps * d, x, y)[0] - tm.loss_and_grad(w - eps * d, x, y)[0]) / (2 * eps)
        assert abs(fd - g @ d) <= 1e-7 * max(1.0, abs(fd)), (fd, g @ d)
    assert loss == pytest.approx(np.mean((tm.forward(w, x) - y) ** 2), rel=1e-14)


def test_product_init_and_oracle_init_agree():
    np.testing.assert_array_equal(lt.xavier(7), tm.xavier_init(7))


def test_bf16_rounding_is_nearest_even():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-3, 5000),
                        [0.0, -0.0, 1.0, 1.00390625, 1.01171875, 3.0e38, 1e-40]]).astype(np.float32)
    # exact ties: halfway between two BF16 values
    ties = (np.arange(1, 200, dtype=np.uint32) << 16 | 0x8000).view(np.float32)
    v = np.concatenate([v, ties, -ties])
    bits, vals = lt.bf16_bits(v)
    ref = torch.from_numpy(v).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    np.testing.assert_array_equal(bits, ref)
    np.testing.assert_array_equal(vals, torch.from_numpy(v).to(torch.bfloat16).float().numpy())


def _net_and_stats(seed=0):
    rng = np.random.default_rng(seed)
    w = lt.bf16_bits(tm.xavier_init(seed) + rng.normal(0, 0.1, tm.NPARAM))[1]
    mean = np.array([1.0, 0.05, 0.0, 0.0, 0.0, 1e-3], np.float32)
    std = np.array([1e-3, 0.02, 0.5, 0.5, 0.5, 1e-3], np.float32)
    lo = np.array([0.9, 0.0, -1.0, -1.0, -1.0, 0.0], np.float32)
    hi = np.array([1.1, 0.2, 1.0, 1.0, 1.0, 0.05], np.float32)
    stats = np.concatenate([mean, std, lo, hi, [0.002]]).astype(np.float32)
    return w, stats


def test_c_oracle_learned_tau_matches_restatement(oracle):
    w, st = _net_and_stats()
    p = np.concatenate([w.astype(np.float64), st.astype(np.float64)])
    rng = np.random.default_rng(2)
    tau0, cs = 0.52, 0.1
    L = oracle.lib()
    import ctypes as C
    n_inside = 0
    for _ in range(200):
        rho = 1 + rng.uniform(-1e-3, 1e-3)
        ux, uy = rng.uniform(-0.08, 0.08, 2)
        ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1.0])
        ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1.0])
        wk = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
        e = ex * ux + ey * uy
        f = wk * rho * (1 + 3 * e + 4.5 * e * e - 1.5 * (ux * ux + uy * uy)) + rng.normal(0, 2e-4, 9)
        # keep rho, u consistent with f (the node's moments)
        rho = f.sum()
        ux, uy = (f * ex).sum() / rho, (f * ey).sum() / rho
        fp = np.ascontiguousarray(f)
        got = L.orc_learned_tau(fp.ctypes.data_as(C.POINTER(C.c_double)), rho, ux, uy, tau0, cs,
                                p.ctypes.data_as(C.POINTER(C.c_double)))
        x = tm.node_features(f, rho, ux, uy, tau0)
        inside = np.all((x >= st[12:18]) & (x <= st[18:24]))
        n_inside += bool(inside)
        if inside:
            want = tau0 + st[24] * tm.forward(p[:1313], ((x - st[:6]) / st[6:12])[None])[0]
        else:
            want = L.orc_les_tau(fp.ctypes.data_as(C.POINTER(C.c_double)), rho, ux, uy, tau0, cs)
        assert got == pytest.approx(want, rel=1e-12, abs=1e-15)
    assert n_inside > 150  # the network path, not only the fallback, is exercised


def test_training_targets_recover_a_known_eddy_viscosity():
    """A shear layer whose effective stress is 2 rho nu S with a known nu:
    the fitted tau is 3 nu + 1/2 and the direction features are -S/|S|."""
    ny, nx = 24, 32
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    ux = 0.02 + 1e-3 * yy + 2e-5 * xx * yy
    uy = -1e-5 * yy * yy
    rho = np.full((ny, nx), 1.0)
    sxx, sxy, syy = lt.strain(ux, uy)
    nu = 0.004
    snap = np.stack([rho, ux, uy, 2 * rho * nu * sxx, 2 * rho * nu * sxy, 2 * rho * nu * syy])
    mask = np.ones((ny, nx), bool)
    tau0 = 0.501
    x, y = lt.samples_from_snapshot(snap, tau0, mask)
    np.testing.assert_allclose(y, 3 * nu + 0.5 - tau0, rtol=1e-12)
    fn = np.sqrt(sxx ** 2 + 2 * sxy ** 2 + syy ** 2).reshape(-1)
    np.testing.assert_allclose(x[:, 3], -sxy.reshape(-1) / fn, rtol=1e-12)
    # |S| feature: the tau0-based estimate at a node relaxed with the target tau
    np.testing.assert_allclose(x[:, 5], (3 * nu + 0.5) / tau0 * np.sqrt(2) * fn, rtol=1e-12)
    # negative fitted viscosity clamps to tau0 (offset 0)
    snap[3:] *= -1
    _, y2 = lt.samples_from_snapshot(snap, tau0, mask)
    assert np.all(y2 == 0)
