"""Precision studies of the benchmark configurations on the GPU.

config2_precision  4096 x 1024, D = 128, Re 3900, MRT and RR + Smagorinsky:
                   FP32 against an FP64 run of the same (mean Cd / Cl, St,
                   L2 of the time-averaged velocity field).
config3_precision  16384 x 4096 (67 M nodes), 64 seeded cylinders D = 48
                   (non-overlapping, gap >= 2 D), Re 1000, MRT + Smagorinsky:
                   FP32 / FP16 / BF16 storage against FP64 (per-cylinder mean
                   Cd, time-averaged velocity L2, mass drift).
The FP64 GPU path is the reference here: it is pinned to the FP64 CPU oracle
bit-for-bit-close (1e-11) by the parity tests, and unlike the CPU oracle it
runs the full lattices.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import _lib as L
from . import scenes
from .lattice import Lattice
from .learned_tau import strouhal


def _run(nx, ny, params, init, markers, ds, bodies, steps, avg_from, chunk=4000):
    lat = Lattice(nx, ny, **dict(params, avg_start=avg_from))
    lat.init_macros(*init)
    lat.set_markers(markers, ds=ds, body=bodies)
    _, m0 = lat.forces(with_mass=True)
    nb = int(bodies.max()) + 1 if bodies is not None else 1
    forces = np.zeros((steps, nb, 2))
    t = 1
    t0 = time.perf_counter()
    while t <= steps:
        n = min(chunk, steps - t + 1)
        lat.step(n, t)
        forces[t - 1:t - 1 + n] = lat.force_history(n)
        t += n
    wall = time.perf_counter() - t0
    _, m1 = lat.forces(with_mass=True)
    avg = np.stack([lat.download(L.FIELD_AVG_U), lat.download(L.FIELD_AVG_V)])
    lat.close()
    return dict(forces=forces, mass0=m0, mass1=m1, avg=avg, wall_s=wall)


def _l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def config2_precision(steps=160000, avg=64000, collisions=(L.MRT, L.RR), log=None):
    out = {}
    for coll in collisions:
        runs = {}
        for st, name in ((L.F64, "f64"), (L.F32, "f32")):
            sc = scenes.config2(collision=coll, storage=st)
            r = _run(sc["nx"], sc["ny"], sc["params"], sc["init"], sc["markers"], sc["ds"], None,
                     steps, steps - avg + 1)
            q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
            f = r["forces"][steps - avg:, 0] / q
            runs[name] = dict(cd=float(f[:, 0].mean()), cl=float(f[:, 1].mean()),
                              st=strouhal(f[:, 1], sc["d"], sc["u_ref"]), avg=r["avg"], wall_s=r["wall_s"])
            if log:
                log(f"config2 {'MRT' if coll == L.MRT else 'RR'} {name}: Cd {runs[name]['cd']:.5f} "
                    f"St {runs[name]['st']:.4f} ({r['wall_s']:.1f} s)")
        a, b = runs["f32"], runs["f64"]
        out["MRT" if coll == L.MRT else "RR"] = dict(
            cd_f64=b["cd"], cd_f32=a["cd"], cd_rel_err=abs(a["cd"] - b["cd"]) / abs(b["cd"]),
            cl_f64=b["cl"], cl_f32=a["cl"], st_f64=b["st"], st_f32=a["st"],
            mean_velocity_l2=_l2(a["avg"], b["avg"]), wall_s_f64=b["wall_s"], wall_s_f32=a["wall_s"])
    return out


def config2_seeds(seeds=(0, 1, 2), steps=480000, avg=400000, collision=L.MRT, log=None):
    """Configuration 2 (4096 x 1024, D = 128, Re 3900, MRT + Smagorinsky) in
    FP32 and FP64 from several seeds of the +-1e-4 initial noise: per seed and
    precision the mean Cd, mean Cl, Cl rms and St over the last `avg` steps.
    The wake is chaotic, so the FP32-FP64 difference of one seed is set
    against the spread between seeds of the same precision."""
    per = {"f32": [], "f64": []}
    for seed in seeds:
        for st, name in ((L.F64, "f64"), (L.F32, "f32")):
            sc = scenes.config2(collision=collision, storage=st, seed=seed)
            r = _run(sc["nx"], sc["ny"], sc["params"], sc["init"], sc["markers"], sc["ds"], None, steps,
                     steps - avg + 1)
            q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
            f = r["forces"][steps - avg:, 0] / q
            rec = dict(seed=int(seed), cd=float(f[:, 0].mean()), cl=float(f[:, 1].mean()),
                       cl_rms=float(f[:, 1].std()), st=strouhal(f[:, 1], sc["d"], sc["u_ref"]),
                       wall_s=r["wall_s"])
            per[name].append(rec)
            if log:
                log(f"config2 seed {seed} {name}: Cd {rec['cd']:.5f} Cl {rec['cl']:+.4f} St {rec['st']:.4f} "
                    f"({r['wall_s']:.1f} s)")

    def spread(v):
        v = np.asarray(v, dtype=np.float64)
        return dict(mean=float(v.mean()), std=float(v.std(ddof=1)) if len(v) > 1 else 0.0,
                    min=float(v.min()), max=float(v.max()))

    out = dict(steps=steps, avg=avg, seeds=[int(s) for s in seeds], runs=per)
    for name in ("f32", "f64"):
        out[name] = {k: spread([r[k] for r in per[name]]) for k in ("cd", "cl", "cl_rms", "st")}
    gaps = [abs(a["cd"] - b["cd"]) / b["cd"] for a, b in zip(per["f32"], per["f64"])]
    out["cd_f32_vs_f64_same_seed"] = dict(per_seed=gaps, mean=float(np.mean(gaps)))
    out["cd_seed_spread_f64"] = out["f64"]["cd"]["std"] / out["f64"]["cd"]["mean"]
    out["cd_mean_f32_vs_f64"] = abs(out["f32"]["cd"]["mean"] - out["f64"]["cd"]["mean"]) / out["f64"]["cd"]["mean"]
    return out


def seeded_cylinders(nx, ny, d, n, gap, seed=0, margin=None):
    """n non-overlapping cylinder centres (centre distance >= d + gap), at
    least `margin` from the lattice edges (default 2 d) and from the inlet
    and outlet (3 d)."""
    rng = np.random.default_rng(seed)
    margin = 2 * d if margin is None else margin
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place the cylinders")
        c = (rng.uniform(3 * d, nx - 3 * d), rng.uniform(margin, ny - margin))
        if all(math.hypot(c[0] - p[0], c[1] - p[1]) >= d + gap for p in pts):
            pts.append(c)
    return np.array(pts)


def config3_scene(nx=16384, ny=4096, d=48, n=64, re=1000.0, u=0.04, seed=0, collision=L.MRT,
                  storage=L.F32):
    centres = seeded_cylinders(nx, ny, d, n, 2 * d, seed)
    sc = scenes.cylinder_channel(nx, ny, d, centres[0, 0], centres[0, 1], u, re, collision=collision,
                                 storage=storage, seed=seed)
    xs, dss, bodies = [], [], []
    for b, (cx, cy) in enumerate(centres):
        xy, ds = scenes.cylinder_markers(cx, cy, d)
        xs.append(xy)
        dss.append(ds)
        bodies.append(np.full(len(ds), b, dtype=np.int32))
    sc.update(markers=np.concatenate(xs), ds=np.concatenate(dss), bodies=np.concatenate(bodies),
              centres=centres)
    return sc


def config3_crop_window(nx=16384, ny=4096, d=48, n=64, seed=0, cw=2048, ch=512, step=64):
    """The cw x ch window of the precision-sweep layout that holds the most
    whole cylinders with the scene's margins (3 d from its inlet and outlet,
    2 d from its walls), scanning x0, y0 on a `step` grid in order; returns
    (x0, y0, centres relative to the window)."""
    c = seeded_cylinders(nx, ny, d, n, 2 * d, seed)
    best = None
    for x0 in range(0, nx - cw + 1, step):
        for y0 in range(0, ny - ch + 1, step):
            r = c - np.array([x0, y0], dtype=np.float64)
            ok = ((r[:, 0] >= 3 * d) & (r[:, 0] <= cw - 3 * d) & (r[:, 1] >= 2 * d) & (r[:, 1] <= ch - 2 * d))
            if best is None or int(ok.sum()) > best[0]:
                best = (int(ok.sum()), x0, y0, r[ok])
    return best[1], best[2], best[3]


def config3_crop_scene(storage=L.F32, cw=2048, ch=512, d=48, re=1000.0, u=0.04, seed=0):
    """A 2048 x 512 crop of the precision-sweep geometry: the cylinders of
    config3_crop_window at their positions in the window, as a channel of
    its own (inlet, outlet and walls at the window's edges), MRT +
    Smagorinsky, Re 1000, the same seeded initial fields as every scene."""
    x0, y0, centres = config3_crop_window(d=d, seed=seed, cw=cw, ch=ch)
    sc = scenes.cylinder_channel(cw, ch, d, centres[0, 0], centres[0, 1], u, re, storage=storage, seed=seed)
    xs, dss, bodies = [], [], []
    for b, (cx, cy) in enumerate(centres):
        xy, ds = scenes.cylinder_markers(cx, cy, d)
        xs.append(xy)
        dss.append(ds)
        bodies.append(np.full(len(ds), b, dtype=np.int32))
    sc.update(markers=np.concatenate(xs), ds=np.concatenate(dss), bodies=np.concatenate(bodies),
              centres=centres, window=(x0, y0))
    return sc


def config3_precision(nx=16384, ny=4096, steps=20000, avg=10000, storages=("f64", "f32", "f16", "bf16"),
                      log=None):
    st_of = {"f64": L.F64, "f32": L.F32, "f16": L.F16, "bf16": L.BF16}
    runs = {}
    for name in storages:
        sc = config3_scene(nx, ny, storage=st_of[name])
        r = _run(nx, ny, sc["params"], sc["init"], sc["markers"], sc["ds"], sc["bodies"], steps,
                 steps - avg + 1)
        q = 0.5 * sc["u_ref"] ** 2 * sc["d"]
        cd = r["forces"][steps - avg:, :, 0].mean(0) / q
        runs[name] = dict(cd=cd, avg=r["avg"], mass_drift=(r["mass1"] - r["mass0"]) / r["mass0"],
                          wall_s=r["wall_s"])
        if log:
            log(f"config3 {name}: mean Cd {cd.mean():.5f}, mass drift {runs[name]['mass_drift']:.3e}, "
                f"{r['wall_s']:.1f} s")
    ref = runs["f64"]
    out = dict(nx=nx, ny=ny, steps=steps, cylinders=int(len(ref["cd"])), f64_mean_cd=float(ref["cd"].mean()),
               f64_mass_drift=ref["mass_drift"], f64_wall_s=ref["wall_s"])
    for name in storages:
        if name == "f64":
            continue
        r = runs[name]
        rel = np.abs(r["cd"] - ref["cd"]) / np.abs(ref["cd"])
        out[name] = dict(cd_rel_err_max=float(rel.max()), cd_rel_err_mean=float(rel.mean()),
                         mean_velocity_l2=_l2(r["avg"], ref["avg"]), mass_drift=r["mass_drift"],
                         wall_s=r["wall_s"],
                         mlups=nx * ny * steps / r["wall_s"] / 1e6)
    return out
