"""ippi_mass_noalloc: the mass checksum for callers that cannot allocate
device memory (under another allocator's ownership of the GPU's memory, in
allocation-free loops).  It must give the mass that
ippi_forces() gives through a lattice handle, on two calls in a row (the
second call reuses the library's fixed scratch array), and refuse fields
taller than its scratch.

This file sorts last so that a run stopping at the first failure has run
every other test before it.  The test allocates its own device buffers
(the entry point does not); it works alone in a fresh process and after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ip = pytest.importorskip("ippi_lbm")
from ippi_lbm import _lib  # noqa: E402


def mass_noalloc(rho_dev, nx, ny, out_dev, stream=None):
    L = ip.lib()
    L.ippi_mass_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    L.ippi_mass_noalloc.restype = C.c_int
    return L.ippi_mass_noalloc(rho_dev, nx, ny, out_dev, stream)


def test_mass_noalloc_matches_handle_mass_twice():
    import torch

    nx, ny = 700, 300
    for call in range(2):
        lat = ip.Lattice(nx, ny, storage=ip.F32, collision=ip.MRT, bc_set=ip.BC_CHANNEL,
                         u_in=0.05, tau0=0.55, cs=0.1)
        rng = np.random.default_rng(call)
        rho0 = 1.0 + rng.uniform(-1e-3, 1e-3, (ny, nx))
        lat.init_macros(rho0, np.zeros((ny, nx)), np.zeros((ny, nx)))
        lat.step(10 + 7 * call, 1)
        _, mass_handle = lat.forces(with_mass=True)
        rho = lat.download(ip.FIELD_RHO)
        rho_dev = torch.from_numpy(rho).cuda()
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = mass_noalloc(rho_dev.data_ptr(), nx, ny, out.data_ptr())
        assert rc == _lib.IPPI_OK
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - mass_handle) <= 1e-13 * abs(mass_handle), (call, got, mass_handle)
        assert abs(got - float(rho.sum())) <= 1e-12 * abs(got)
        lat.close()


def test_mass_noalloc_rejects_fields_taller_than_its_scratch():
    import torch

    ny = _lib_max_rows() + 1
    rho_dev = torch.ones((ny, 4), dtype=torch.float64, device="cuda")
    out = torch.zeros((1,), dtype=torch.float64, device="cuda")
    assert mass_noalloc(rho_dev.data_ptr(), 4, ny, out.data_ptr()) == _lib.IPPI_ERR_ARG
    assert mass_noalloc(rho_dev.data_ptr(), 4, ny - 1, out.data_ptr()) == _lib.IPPI_OK
    torch.cuda.synchronize()
    assert float(out.item()) == 4.0 * (ny - 1)


def _lib_max_rows():
    import os
    import re

    from conftest import REPO

    src = open(os.path.join(REPO, "include", "ippi_lbm.h")).read()
    return int(re.search(r"#define IPPI_NOALLOC_MAX_ROWS (\d+)", src).group(1))
