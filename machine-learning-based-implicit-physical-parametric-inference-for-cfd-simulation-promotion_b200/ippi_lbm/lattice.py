"""Lattice: a Python handle on one ippi_lbm lattice (thin, over the C ABI)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L


def _f64(a, n=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def _p(a, ct=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


class Lattice:
    """One D2Q9 lattice on the GPU.  Keyword arguments fill ippi_params
    (defaults: the reference's main.cpp constants for the given size)."""

    def __init__(self, nx, ny, **kw):
        p = L.Params()
        L.lib().ippi_params_default(C.byref(p), nx, ny)
        for k, v in kw.items():
            if not hasattr(p, k):
                raise TypeError(f"unknown parameter {k}")
            setattr(p, k, v)
        self.params = p
        self.nx, self.ny = nx, ny
        h = C.c_void_p()
        L.check(L.lib().ippi_create(C.byref(p), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            L.lib().ippi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def init_macros(self, rho=None, ux=None, uy=None):
        n = self.nx * self.ny
        rho, ux, uy = _f64(rho, n), _f64(ux, n), _f64(uy, n)
        L.check(L.lib().ippi_init_macros(self._h, _p(rho), _p(ux), _p(uy)), self._h)

    def init_macros_f32(self, rho=None, ux=None, uy=None):
        """init_macros from FP32 arrays (ippi_init_macros_f32); float32
        C-contiguous arrays are passed without a copy."""
        n = self.nx * self.ny

        def f32(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            if a.size != n:
                raise ValueError(f"expected {n} values, got {a.size}")
            return a
        rho, ux, uy = f32(rho), f32(ux), f32(uy)
        L.check(L.lib().ippi_init_macros_f32(self._h, _p(rho, C.c_float), _p(ux, C.c_float),
                                             _p(uy, C.c_float)), self._h)

    def download_f32(self, field, out=None):
        """A field rounded to FP32 (ippi_download_f32), into `out` when given."""
        shape = (9, self.ny, self.nx) if field == L.FIELD_F else (self.ny, self.nx)
        if out is None:
            out = np.zeros(shape, np.float32)
        L.check(L.lib().ippi_download_f32(self._h, field, _p(out, C.c_float), out.nbytes), self._h)
        return out

    def reequilibrate(self, rho=None, ux=None, uy=None):
        """Populations at the equilibrium of the given moments, keeping the
        running means and the force history (a step must have been taken)."""
        n = self.nx * self.ny
        rho, ux, uy = _f64(rho, n), _f64(ux, n), _f64(uy, n)
        L.check(L.lib().ippi_reequilibrate(self._h, _p(rho), _p(ux), _p(uy)), self._h)

    def set_markers(self, xy, ub=None, body=None, ds=None):
        xy = _f64(xy).reshape(-1)
        n = xy.size // 2
        ub = _f64(ub, 2 * n)
        ds = _f64(ds, n)
        bd = None if body is None else np.ascontiguousarray(body, dtype=np.int32)
        L.check(L.lib().ippi_set_markers(self._h, n, _p(xy), _p(ub),
                                         None if bd is None else bd.ctypes.data_as(C.POINTER(C.c_int)),
                                         _p(ds)), self._h)

    def load_band_net(self, t, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        L.check(L.lib().ippi_load_band_net(self._h, t, _p(w, C.c_float), w.size), self._h)

    def step(self, n=1, t0=1):
        L.check(L.lib().ippi_step(self._h, n, t0), self._h)

    def set_learned_tensor_cores(self, on=True):
        """The learned tau's hidden layer on the tensor cores (BF16 mma.sync,
        FP32 accumulation) or on FP32 FMA (ippi_set_learned_tensor_cores)."""
        L.check(L.lib().ippi_set_learned_tensor_cores(self._h, int(bool(on))), self._h)

    def set_les_cs(self, cs):
        """Smagorinsky constant of the following steps (ippi_set_les_cs)."""
        L.check(L.lib().ippi_set_les_cs(self._h, float(cs)), self._h)
        self.params.cs = float(cs)

    def step_timed(self, n, t0=1):
        """step() with device timing: milliseconds between CUDA events on the
        handle's stream around the n steps, queued behind a short hold so
        they run back to back (ippi_step_timed)."""
        ms = C.c_double()
        L.check(L.lib().ippi_step_timed(self._h, n, t0, C.byref(ms)), self._h)
        return ms.value

    def profile_steps(self, n, t0=1):
        b, nb, ib = C.c_double(), C.c_double(), C.c_double()
        L.check(L.lib().ippi_profile_steps(self._h, n, t0, C.byref(b), C.byref(nb), C.byref(ib)),
                self._h)
        return b.value, nb.value, ib.value

    def download(self, field):
        if field == L.FIELD_FLAGS:
            out = np.zeros((self.ny, self.nx), np.uint8)
        elif field == L.FIELD_F:
            out = np.zeros((9, self.ny, self.nx), np.float64)
        else:
            out = np.zeros((self.ny, self.nx), np.float64)
        L.check(L.lib().ippi_download(self._h, field, out.ctypes.data_as(C.c_void_p), out.nbytes),
                self._h)
        return out

    def forces(self, with_mass=False):
        nb = C.c_int(0)
        L.check(L.lib().ippi_forces(self._h, None, C.byref(nb), None), self._h)
        f = np.zeros(max(2 * nb.value, 2))
        m = C.c_double(0)
        L.check(L.lib().ippi_forces(self._h, _p(f), C.byref(nb), C.byref(m) if with_mass else None),
                self._h)
        f = f[: 2 * nb.value].reshape(-1, 2)
        return (f, m.value) if with_mass else f

    def force_history(self, max_steps):
        nb = C.c_int(0)
        L.check(L.lib().ippi_forces(self._h, None, C.byref(nb), None), self._h)
        out = np.zeros((max_steps, max(nb.value, 1), 2))
        n = L.lib().ippi_force_history(self._h, _p(out), max_steps)
        if n < 0:
            L.check(n, self._h)
        return out[:n, : nb.value]

    def load_tau_mlp(self, w_bf16, stats):
        """Learned relaxation time: w_bf16[1313] BF16 bit patterns (uint16),
        stats[25] (mean, std, lo, hi of the 6 features, out_scale)."""
        w = np.ascontiguousarray(w_bf16, dtype=np.uint16)
        st = np.ascontiguousarray(stats, dtype=np.float32)
        L.check(L.lib().ippi_load_tau_mlp(self._h, w.ctypes.data_as(C.POINTER(C.c_uint16)), w.size,
                                          st.ctypes.data_as(C.POINTER(C.c_float)), st.size), self._h)

    def load_tau_mlp_f32(self, w, stats):
        """Learned tau with FP32 weights used as given (no BF16 rounding)."""
        w = np.ascontiguousarray(w, dtype=np.float32)
        st = np.ascontiguousarray(stats, dtype=np.float32)
        L.check(L.lib().ippi_load_tau_mlp_f32(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size,
                                              st.ctypes.data_as(C.POINTER(C.c_float)), st.size), self._h)

    def set_tau_field(self, tau):
        """Relaxation time per node [ny][nx] for les_model = LES_FIELD."""
        tau = _f64(tau, self.nx * self.ny)
        L.check(L.lib().ippi_set_tau_field(self._h, _p(tau)), self._h)

    def adjoint_forward(self, nsteps, t0=1, ckpt_every=64):
        """Advance nsteps steps, recording checkpoints for adjoint_backward."""
        L.check(L.lib().ippi_adjoint_forward(self._h, nsteps, t0, ckpt_every), self._h)

    def adjoint_backward(self, dl_dforce=None, dl_dmacro=None, tau=False, mlp=False, f0=False):
        """Gradients of the loss with partial derivatives dl_dforce
        [nsteps][nbody][2] and dl_dmacro [3][ny][nx] (final post-stream rho,
        ux, uy): dict with 'tau' [ny][nx], 'mlp' [1313], 'f0' [9][ny][nx]."""
        nn = self.nx * self.ny
        dF = None if dl_dforce is None else _f64(dl_dforce)
        dM = None if dl_dmacro is None else _f64(dl_dmacro, 3 * nn)
        out = {}
        gt = np.zeros((self.ny, self.nx)) if tau else None
        gm = np.zeros(L.MLP_PARAMS) if mlp else None
        gf = np.zeros((9, self.ny, self.nx)) if f0 else None
        L.check(L.lib().ippi_adjoint_backward(self._h, _p(dF), _p(dM), _p(gt), _p(gm), _p(gf)), self._h)
        if tau:
            out["tau"] = gt
        if mlp:
            out["mlp"] = gm
        if f0:
            out["f0"] = gf
        return out

    def set_wall_distance(self, dist):
        """Wall distance per node [ny][nx] for the wall-damped closure."""
        d = _f64(dist, self.nx * self.ny)
        L.check(L.lib().ippi_set_wall_distance(self._h, _p(d)), self._h)

    def diagnostics(self):
        """dict(max_u, net_nodes, fallback_nodes) of the state after the last
        step (ippi_diagnostics)."""
        mu, net, fb = C.c_double(), C.c_longlong(), C.c_longlong()
        L.check(L.lib().ippi_diagnostics(self._h, C.byref(mu), C.byref(net), C.byref(fb)), self._h)
        return dict(max_u=mu.value, net_nodes=net.value, fallback_nodes=fb.value)

    def save_state(self, path=None):
        """Checkpoint of the evolving state (ippi_save_state) as bytes; also
        written to `path` when given."""
        n = C.c_size_t()
        L.check(L.lib().ippi_state_bytes(self._h, C.byref(n)), self._h)
        buf = np.empty(n.value, dtype=np.uint8)
        L.check(L.lib().ippi_save_state(self._h, buf.ctypes.data_as(C.c_void_p), buf.nbytes), self._h)
        if path is not None:
            buf.tofile(path)
        return buf.tobytes()

    def load_state(self, data):
        """Restore a checkpoint (bytes, or a file path); returns the user step
        number of its last step (stepping resumes at that + 1)."""
        if isinstance(data, (str, os.PathLike)):
            buf = np.fromfile(data, dtype=np.uint8)
        else:
            buf = np.frombuffer(bytes(data), dtype=np.uint8).copy()
        last = C.c_int()
        L.check(L.lib().ippi_load_state(self._h, buf.ctypes.data_as(C.c_void_p), buf.nbytes, C.byref(last)),
                self._h)
        return last.value

    def set_solid(self, mask):
        """Solid nodes: mask[ny][nx] (nonzero = solid); None removes them."""
        if mask is None:
            L.check(L.lib().ippi_set_solid(self._h, None, 0), self._h)
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        L.check(L.lib().ippi_set_solid(self._h, m.ctypes.data_as(C.POINTER(C.c_uint8)), m.size), self._h)

    def solid_force(self):
        """Momentum-exchange force (Fx, Fy) on the solids after the last step."""
        out = np.zeros(2)
        L.check(L.lib().ippi_solid_force(self._h, _p(out)), self._h)
        return out

    def tau_scan(self, xy, target, m_lo=-10000, m_hi=10000, step=1e-5):
        """Mesh::FindAndWriteTau's scan at the current state: best dtau and
        its error for interior nodes xy[n][2] and targets target[n][3]."""
        xy = np.ascontiguousarray(xy, dtype=np.int32).reshape(-1, 2)
        target = _f64(target).reshape(-1, 3)
        n = xy.shape[0]
        bd, be = np.zeros(n), np.zeros(n)
        L.check(L.lib().ippi_tau_scan(self._h, n, xy.ctypes.data_as(C.POINTER(C.c_int)), _p(target), m_lo,
                                      m_hi, step, _p(bd), _p(be)), self._h)
        return bd, be

    def filter_snapshot(self, factor):
        """Box-filtered state [6][ny/f][nx/f]: rho, ux, uy (density-weighted),
        effective stress Sxx, Sxy, Syy (include/ippi_lbm.h)."""
        out = np.zeros((6, self.ny // factor, self.nx // factor))
        L.check(L.lib().ippi_filter_snapshot(self._h, factor, _p(out), out.nbytes), self._h)
        return out

    def stream(self) -> int:
        s = C.c_void_p()
        L.check(L.lib().ippi_get_stream(self._h, C.byref(s)), self._h)
        return s.value or 0
