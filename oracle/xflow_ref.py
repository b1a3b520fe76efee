"""Restatement of the reference's XFlow import (TEST INFRASTRUCTURE ONLY:
used by tests/ as the checker of the host reader, never by the product).

Mesh::ReadXflowdata / ManageDataFromXflow (IPPI-LBM/mesh.cpp:2189-2547) and
RoundToThreeDecimalPlaces (mesh.cpp:41-46), in plain Python on the same
double arithmetic:
  * header line skipped; a data line needs 13 numbers, each followed by one
    separator (id, x, y, z, VelocityModule, StaticPressure, -, TotalPressure,
    -, viscosity, ux, uy, uz), else it is skipped (mesh.cpp:2222-2236);
  * x, y rounded half away from zero to 1e-3; x -> (x + 0.4) / 0.001,
    y, z -> / 0.001; velocities -> v / 340.112 / sqrt(3); TotalPressure ->
    (StaticPressure + 101325) / 101325 (mesh.cpp:2271-2287);
  * equal (x, y): (kept + new) / 2 for every other field (mesh.cpp:2291-2322);
  * x outside [lo - 0.5, hi + 0.5] of the rank dropped (mesh.cpp:2348-2360).
"""
import math

FIELDS = ("id", "vx", "vy", "vz", "VelocityModule", "StaticPress", "-", "TotalPressure", "-",
          "viscosity", "ux", "uy", "uz")
MERGED = ("VelocityModule", "StaticPress", "TotalPressure", "ux", "uy", "uz", "vz", "viscosity")


def _round3(v):
    t = v * 1000.0
    r = math.floor(t + 0.5) if t >= 0 else -math.floor(-t + 0.5)
    return r / 1000.0


def _parse(line):
    parts = line.split(",")
    if len(parts) < 14:
        return None
    try:
        vals = [float(p) for p in parts[:13]]
    except ValueError:
        return None
    return {k: v for k, v in zip(FIELDS, vals) if k not in ("id", "-")}


def read(path):
    with open(path) as f:
        lines = f.read().splitlines()
    out, where = [], {}
    for line in lines[1:]:
        p = _parse(line)
        if p is None:
            continue
        p["vx"] = (_round3(p["vx"]) + 0.4) / 0.001
        p["vy"] = _round3(p["vy"]) / 0.001
        p["vz"] = p["vz"] / 0.001
        for k in ("VelocityModule", "ux", "uy", "uz"):
            p[k] = p[k] / 340.112 / math.sqrt(3.0)
        p["TotalPressure"] = (p["StaticPress"] + 101325) / 101325
        key = (p["vx"], p["vy"])
        if key in where:
            kept = out[where[key]]
            for k in MERGED:
                kept[k] = (kept[k] + p[k]) / 2.0
        else:
            where[key] = len(out)
            out.append(p)
    return out


def clip(points, nx_total, rank=0, ncore=1, parallel_size=None):
    parallel_size = nx_total if parallel_size is None else parallel_size
    lo, hi = rank * parallel_size, (rank + 1) * parallel_size + 2
    if rank == ncore - 1:
        hi = nx_total
    if rank == 0:
        lo -= 2
    return [p for p in points if not (p["vx"] < lo - 0.5 or p["vx"] > hi + 0.5)]


def node_of(p, nx, ny):
    """(x, y) of the node the point lands on (|vx - x| < 1e-3, |vy - y| < 1e-3), or None."""
    rx, ry = round(p["vx"]), round(p["vy"])
    if abs(p["vx"] - rx) < 0.001 and abs(p["vy"] - ry) < 0.001 and 0 <= rx < nx and 0 <= ry < ny:
        return int(rx), int(ry)
    return None
