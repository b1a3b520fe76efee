"""The bounded wait of the one-launch step's IB barrier, tested without a GPU
fault: in a child process the test knob IPPI_TEST_IB_BARRIER_EXTRA=1 makes
every barrier wait for an arrival that never comes.  Each wait must give up
after about a second, the step must report the timeout, and the GPU context
must stay usable (a lattice without markers steps and downloads afterwards)."""
import os
import subprocess
import sys
import textwrap

import pytest

from conftest import PKG_DIR

pytestmark = pytest.mark.gpu

CHILD = textwrap.dedent("""
    import sys, time
    sys.path.insert(0, %r)
    import numpy as np
    import ippi_lbm as ip
    from ippi_lbm import scenes
    sc = scenes.cylinder_channel(128, 64, 10, 40.3, 31.7, 0.05, 100)
    g = ip.Lattice(128, 64, **sc["params"])
    g.set_markers(sc["markers"], ds=sc["ds"])
    g.init_macros(*sc["init"])
    t0 = time.perf_counter()
    try:
        g.step(1, 1)
        print("NO-ERROR")
    except ip.IppiError as e:
        print("ERROR", time.perf_counter() - t0, e)
    g.close()
    h = ip.Lattice(128, 64, **sc["params"])
    h.init_macros(*sc["init"])
    h.step(10, 1)
    print("AFTER", float(np.abs(h.download(ip.FIELD_UX)).max()))
""") % PKG_DIR


def test_ib_barrier_timeout_is_reported_and_context_survives():
    env = dict(os.environ, IPPI_TEST_IB_BARRIER_EXTRA="1")
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    out = r.stdout
    err = [ln for ln in out.splitlines() if ln.startswith("ERROR")]
    assert err and "barrier timed out" in err[0], out
    secs = float(err[0].split()[1])
    assert 2.0 < secs < 30.0, secs  # three barriers of about 1 s each
    after = [ln for ln in out.splitlines() if ln.startswith("AFTER")]
    assert after and 0.0 < float(after[0].split()[1]) < 0.2, out
