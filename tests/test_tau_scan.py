"""Implicit tau inference (Mesh::FindAndWriteTau, mesh.cpp:2625-2715): the
oracle's restatement against a brute-force numpy scan and a planted answer
(CPU), and the GPU warp-parallel scan against the oracle bit for bit (GPU)."""
import numpy as np
import pytest

import pyoracle as po

EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])


def plate_state(oracle):
    o = oracle.Oracle(64, 16, collision=oracle.BGK, tau0=0.55, cs=0.173, u_in=0.1, plate_x0=20)
    rng = np.random.default_rng(0)
    o.init_macros(1 + rng.uniform(-1e-3, 1e-3, (16, 64)), 0.08 + rng.uniform(-1e-2, 1e-2, (16, 64)),
                  rng.uniform(-1e-2, 1e-2, (16, 64)))
    o.step(15, 1)
    f = o.get(po.F)
    m3 = np.stack([o.get(po.RHO), o.get(po.UX), o.get(po.UY)])
    return f, m3, o.get(po.TAU)


def numpy_scan(f, m3, tau, x, y, target, m_lo, m_hi, step):
    fn, fe, tn = [], [], []
    for k in range(9):
        sx, sy = x - EX[k], y - EY[k]
        r, u, v = m3[0, sy, sx], m3[1, sy, sx], m3[2, sy, sx]
        eu = EX[k] * u + EY[k] * v
        w = [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4
        fe.append(w[k] * r * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * (u * u + v * v)))
        fn.append(f[k, sy, sx])
        tn.append(tau[sy, sx])
    m = np.arange(m_lo, m_hi + 1)
    d = m * step
    c = np.stack([(1 - 1 / (tn[k] + d)) * fn[k] + fe[k] / (tn[k] + d) for k in range(9)])
    err = (np.abs(c.sum(0) - target[0]) + np.abs((c * EX[:, None]).sum(0) - target[1])
           + np.abs((c * EY[:, None]).sum(0) - target[2]))
    i = int(np.argmin(err))  # first minimum
    return d[i], err[i], c[:, i]


def test_oracle_scan_matches_brute_force_and_recovers_a_planted_tau(oracle):
    f, m3, tau = plate_state(oracle)
    rng = np.random.default_rng(1)
    xy = np.array([[10, 5], [33, 8], [50, 12]])
    # planted: the target is what dtau* = 0.01234 produces
    tg = []
    for x, y in xy:
        _, _, c = numpy_scan(f, m3, tau, x, y, np.zeros(3), 1234, 1234, 1e-5)
        tg.append([c.sum(), (c * EX).sum(), (c * EY).sum()])
    tg = np.array(tg)
    bd, be = po.tau_scan_state(f, m3, tau, xy, tg)
    np.testing.assert_allclose(bd, 0.01234, rtol=0, atol=1e-12)
    assert np.all(be < 1e-13)
    # random targets near the state: the same first minimum as numpy
    tg2 = tg + rng.normal(0, 1e-4, tg.shape)
    bd2, be2 = po.tau_scan_state(f, m3, tau, xy, tg2, -3000, 3000, 1e-5)
    for q, (x, y) in enumerate(xy):
        d, e, _ = numpy_scan(f, m3, tau, x, y, tg2[q], -3000, 3000, 1e-5)
        assert bd2[q] == pytest.approx(d, abs=1e-12) and be2[q] == pytest.approx(e, rel=1e-9)


@pytest.mark.gpu
def test_gpu_scan_equals_oracle_bit_for_bit(oracle):
    torch = pytest.importorskip("torch")
    import ippi_lbm as ip
    from ippi_lbm import _lib

    f, m3, tau = plate_state(oracle)
    rng = np.random.default_rng(2)
    xy = np.stack([rng.integers(1, 63, 300), rng.integers(1, 15, 300)], 1).astype(np.int32)
    tg = np.stack([m3[0][xy[:, 1], xy[:, 0]], m3[1][xy[:, 1], xy[:, 0]], m3[2][xy[:, 1], xy[:, 0]]], 1)
    tg = tg + rng.normal(0, 2e-4, tg.shape)
    want_d, want_e = po.tau_scan_state(f, m3, tau, xy, tg)
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (f, m3, tau, xy, tg)]
    out = torch.zeros((2, 300), dtype=torch.float64, device=dev)
    rc = _lib.lib().ippi_tau_scan_state(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), 64, 16, 300,
                                        t[3].data_ptr(), t[4].data_ptr(), -10000, 10000, 1e-5,
                                        out[0].data_ptr(), out[1].data_ptr(),
                                        torch.cuda.current_stream(dev).cuda_stream)
    assert rc == 0
    got = out.cpu().numpy()
    assert np.array_equal(got[0], want_d) and np.array_equal(got[1], want_e)
    # through a handle: the lattice's own post-stream state (FP64)
    g = ip.Lattice(64, 16, storage=ip.F64, collision=ip.BGK, tau0=0.55, cs=0.173, u_in=0.1, plate_x0=20)
    r2 = np.random.default_rng(0)
    g.init_macros(1 + r2.uniform(-1e-3, 1e-3, (16, 64)), 0.08 + r2.uniform(-1e-2, 1e-2, (16, 64)),
                  r2.uniform(-1e-2, 1e-2, (16, 64)))
    g.step(15, 1)
    bd, be = g.tau_scan(xy, tg)
    assert np.abs(bd - want_d).max() <= 1e-5 + 1e-12  # same state to ~1e-15: at most one grid step apart
    np.testing.assert_allclose(be, want_e, rtol=1e-6, atol=1e-12)
