"""ctypes bindings for the FP64 oracle and the reference-build checker.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package.

* ``Oracle`` wraps oracle/_build/libippi_oracle.so (built by ``make -C oracle``),
  the FP64 restatement of the reference step (see ippi_oracle.h).
* ``RefSim`` wraps oracle/_ref/libippi_ref_<variant>.so (built by
  oracle/build_ref.sh from the reference sources), the reference's own Mesh
  class driven as main.cpp drives it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libippi_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

F, RHO, UX, UY, TAU, AVG_U, AVG_V, AVG_RHO, FLAGS, NNFLAG = range(10)
BGK, MRT, RR = 0, 1, 2
BC_REF, BC_CHANNEL = 0, 1

_dp = C.POINTER(C.c_double)


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("collision", C.c_int), ("bc_set", C.c_int),
        ("les_model", C.c_int), ("tau0", C.c_double), ("cs", C.c_double),
        ("u_in", C.c_double), ("rho0", C.c_double), ("plate_x0", C.c_int),
        ("avg_start", C.c_int), ("delta_kernel", C.c_int), ("mdf_iters", C.c_int),
    ]


def build_oracle() -> str:
    """Compile the oracle if needed (make is incremental)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return ORACLE_SO


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_threads.restype = C.c_int
        L.orc_init_macros.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_set_markers.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.POINTER(C.c_int), _dp]
        L.orc_load_band_net.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_float), C.c_size_t]
        L.orc_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_get.argtypes = [C.c_void_p, C.c_int, _dp]
        L.orc_forces.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_ib_probe.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_num_bodies.argtypes = [C.c_void_p]
        L.orc_peskin_phi.restype = C.c_double
        L.orc_peskin_phi.argtypes = [C.c_double]
        L.orc_band_forward.restype = C.c_float
        L.orc_band_forward.argtypes = [C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float)]
        L.orc_marker_stencil.argtypes = [C.c_int, C.c_double, C.c_double,
                                         C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]
        L.orc_collide_node.argtypes = [C.c_int, _dp, C.c_double, C.c_double, C.c_double,
                                       C.c_double, _dp]
        L.orc_les_tau.restype = C.c_double
        L.orc_les_tau.argtypes = [_dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_set_tau_field.argtypes = [C.c_void_p, _dp]
        L.orc_set_solid.argtypes = [C.c_void_p, C.POINTER(C.c_uint8)]
        L.orc_set_wall_distance.argtypes = [C.c_void_p, _dp]
        L.orc_solid_force.argtypes = [C.c_void_p, _dp]
        L.orc_tau_scan_state.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_int), _dp, C.c_int, C.c_int, C.c_double,
                                         _dp, _dp]
        L.orc_force_node.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_double, _dp]
        L.orc_load_tau_mlp.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_size_t,
                                       C.POINTER(C.c_float), C.c_size_t]
        L.orc_learned_tau.argtypes = [_dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _dp]
        L.orc_learned_tau.restype = C.c_double
        _lib = L
    return _lib


def _ptr(a, ct=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """FP64 CPU restatement of the reference step on an nx x ny lattice."""

    def __init__(self, nx, ny, collision=BGK, bc_set=BC_REF, les_model=1, tau0=0.6,
                 cs=0.173, u_in=0.1, rho0=1.0, plate_x0=400, avg_start=30000,
                 delta_kernel=1, mdf_iters=1):
        self.nx, self.ny = nx, ny
        p = OrcParams(nx, ny, collision, bc_set, les_model, tau0, cs, u_in, rho0,
                      plate_x0, avg_start, delta_kernel, mdf_iters)
        self._h = lib().orc_create(C.byref(p))
        if not self._h:
            raise ValueError("orc_create rejected the parameters")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def init_macros(self, rho=None, ux=None, uy=None):
        rho, ux, uy = _f64(rho), _f64(ux), _f64(uy)
        lib().orc_init_macros(self._h, _ptr(rho), _ptr(ux), _ptr(uy))

    def set_markers(self, xy, ub=None, body=None, ds=None):
        xy = _f64(xy).reshape(-1)
        n = xy.size // 2
        ub = _f64(ub).reshape(-1) if ub is not None else None
        ds = _f64(ds) if ds is not None else None
        bd = np.ascontiguousarray(body, dtype=np.int32) if body is not None else None
        rc = lib().orc_set_markers(self._h, n, _ptr(xy), _ptr(ub),
                                   None if bd is None else bd.ctypes.data_as(C.POINTER(C.c_int)),
                                   _ptr(ds))
        if rc != 0:
            raise ValueError("marker stencil leaves the interior")

    def load_band_net(self, t, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        rc = lib().orc_load_band_net(self._h, t, _ptr(w, C.c_float), w.size)
        if rc != 0:
            raise ValueError("bad net")

    def load_tau_mlp(self, w, stats):
        """Learned-tau network: w[1313] (FP32 values of the BF16 weights),
        stats[25]."""
        w = np.ascontiguousarray(w, dtype=np.float32)
        st = np.ascontiguousarray(stats, dtype=np.float32)
        if lib().orc_load_tau_mlp(self._h, _ptr(w, C.c_float), w.size, _ptr(st, C.c_float), st.size):
            raise ValueError("bad tau network")

    def set_tau_field(self, tau):
        tau = np.ascontiguousarray(tau, dtype=np.float64)
        lib().orc_set_tau_field(self._h, _ptr(tau))

    def set_wall_distance(self, d):
        d = np.ascontiguousarray(d, dtype=np.float64)
        lib().orc_set_wall_distance(self._h, _ptr(d))

    def set_solid(self, mask):
        m = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        if lib().orc_set_solid(self._h, None if m is None else m.ctypes.data_as(C.POINTER(C.c_uint8))):
            raise ValueError("solid nodes must be at least 3 nodes inside a channel lattice")

    def solid_force(self):
        out = np.zeros(2)
        lib().orc_solid_force(self._h, _ptr(out))
        return out

    def step(self, n, t0=1):
        return lib().orc_step(self._h, n, t0)

    def get(self, field):
        shape = (9, self.ny, self.nx) if field == F else (self.ny, self.nx)
        out = np.zeros(shape, np.float64)
        lib().orc_get(self._h, field, _ptr(out))
        return out

    def forces(self):
        nb = lib().orc_num_bodies(self._h)
        fxy = np.zeros(max(2 * nb, 2), np.float64)
        m = C.c_double(0)
        lib().orc_forces(self._h, _ptr(fxy), C.byref(m))
        return fxy[: 2 * nb].reshape(-1, 2), m.value

    def ib_probe(self, nmark):
        vref = np.zeros(2 * nmark)
        mf = np.zeros(2 * nmark)
        nf = np.zeros((2, self.ny, self.nx))
        lib().orc_ib_probe(self._h, _ptr(vref), _ptr(mf), _ptr(nf))
        return vref.reshape(-1, 2), mf.reshape(-1, 2), nf


# --------------------------------------------------------------------------
# reference build (checker)
# --------------------------------------------------------------------------

REF_VARIANTS = ("srt", "srt_peskin", "mrt", "rr", "srt_f32", "mrt_f32")


def threads() -> int:
    """Threads of the oracle's per-node loops (OpenMP; results do not depend
    on the count)."""
    return int(lib().orc_threads())


def ref_available(variant="srt") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libippi_ref_{variant}.so"))


def build_ref() -> bool:
    """Build oracle/_ref from the reference sources when they are present."""
    script = os.path.join(HERE, "build_ref.sh")
    subprocess.run([script], check=True, stdout=subprocess.DEVNULL)
    return ref_available()


_ref_libs: dict = {}


def ref_lib(variant="srt") -> C.CDLL:
    if variant not in _ref_libs:
        path = os.path.join(REF_DIR, f"libippi_ref_{variant}.so")
        L = C.CDLL(path)
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                 C.c_int, C.c_int]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_init_macros.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.ref_step.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ref_get.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_ib_probe.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double,
                                   _dp, _dp, _dp, _dp]
        _ref_libs[variant] = L
    return _ref_libs[variant]


class RefSim:
    """The reference's Mesh, driven like main.cpp (flat-plate scene)."""

    def __init__(self, nx, ny, tau, cs=0.173, u_in=0.1, avg_start=30000, ranks=1,
                 variant="srt"):
        self.nx, self.ny, self.variant = nx, ny, variant
        if variant.endswith("_torch"):
            # the libtorch build loads the shipped archives copied next to it
            os.environ.setdefault("IPPI_REF_PT_DIR", os.path.join(REF_DIR, "nn"))
        self._L = ref_lib(variant)
        self._h = self._L.ref_create(nx, ny, tau, cs, u_in, avg_start, ranks)

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.ref_destroy(self._h)
            self._h = None

    def init_macros(self, rho=None, ux=None, uy=None):
        rho, ux, uy = _f64(rho), _f64(ux), _f64(uy)
        self._L.ref_init_macros(self._h, _ptr(rho), _ptr(ux), _ptr(uy))

    def step(self, n, t0=1):
        return self._L.ref_step(self._h, n, t0)

    def get(self, field):
        shape = (9, self.ny, self.nx) if field == F else (self.ny, self.nx)
        out = np.zeros(shape, np.float64)
        self._L.ref_get(self._h, field, _ptr(out))
        return out

    def ib_probe(self, n, radius, cx, cy):
        xy = np.zeros(2 * n)
        vref = np.zeros(2 * n)
        mf = np.zeros(2 * n)
        nf = np.zeros((2, self.ny, self.nx))
        rc = self._L.ref_ib_probe(self._h, n, radius, cx, cy, _ptr(xy), _ptr(vref),
                                  _ptr(mf), _ptr(nf))
        if rc != 0:
            raise RuntimeError("ref_ib_probe failed")
        return xy.reshape(-1, 2), vref.reshape(-1, 2), mf.reshape(-1, 2), nf


def tau_scan_state(f, m3, tau, xy, target, m_lo=-10000, m_hi=10000, step=1e-5):
    """Mesh::FindAndWriteTau's scan on a given state (see ippi_oracle.h)."""
    f = np.ascontiguousarray(f, dtype=np.float64)
    m3 = np.ascontiguousarray(m3, dtype=np.float64)
    tau = np.ascontiguousarray(tau, dtype=np.float64)
    xy = np.ascontiguousarray(xy, dtype=np.int32)
    target = np.ascontiguousarray(target, dtype=np.float64)
    n = xy.shape[0]
    ny, nx = tau.shape
    bd, be = np.zeros(n), np.zeros(n)
    lib().orc_tau_scan_state(_ptr(f), _ptr(m3), _ptr(tau), nx, ny, n,
                             xy.ctypes.data_as(C.POINTER(C.c_int)), _ptr(target), m_lo, m_hi, step,
                             _ptr(bd), _ptr(be))
    return bd, be
