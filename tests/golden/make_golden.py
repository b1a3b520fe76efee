"""Generate the committed golden fixtures under tests/golden/.

Run where the reference project is mounted (the root is the argument, else
$IPPI_REFERENCE_DIR, else the reference's mount point /root/reference):

    python tests/golden/make_golden.py [reference-root]

It writes
  band_nets/AutoT0{1,3,5,7}.f32   the shipped boundary nets' parameters, raw
                                  float32 in TorchScript parameter order
                                  (hidden_layer1.weight [128][15], .bias,
                                  hidden_layer2..7, output_layer), read with
                                  torch.jit.load from NNmodel/AutoT0x.pt;
  band_net_golden.npz             seeded inputs and the nets' float32 outputs
                                  computed by torch itself (the pin for the
                                  oracle's and the kernel's forward pass);
  ref_golden.json                 outputs of the reference build
                                  (oracle/build_ref.sh): SHA-256 of every
                                  float64 field plus sampled values, for the
                                  flat-plate step (BGK/MRT/RR, nets on/off)
                                  and for the IB primitives (bilinear, Peskin).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

NET_TYPES = (1, 3, 5, 7)

# Flat-plate cases: the bottom wall switches from specular to NEE no-slip at
# x = 400 (mesh.cpp:1413), so the lattice is 416 wide to contain both parts.
PLATE_CASES = [
    dict(name="plate_bgk", variant="srt", nx=416, ny=12, tau=0.55, cs=0.173, steps=[1, 25],
         nets=False, avg_start=10),
    dict(name="plate_bgk_nets", variant="srt", nx=416, ny=12, tau=0.52, cs=0.173, steps=[1, 20],
         nets=True, avg_start=10),
    dict(name="plate_mrt", variant="mrt", nx=416, ny=12, tau=0.53, cs=0.173, steps=[1, 25],
         nets=False, avg_start=10),
    dict(name="plate_rr", variant="rr", nx=416, ny=12, tau=0.53, cs=0.173, steps=[1, 25],
         nets=False, avg_start=10),
]
IB_CASES = [
    dict(name="ib_bilinear", variant="srt", nx=64, ny=40, tau=0.6, pre_steps=30,
         n=32, radius=5.0, cx=12.3, cy=20.2),
    dict(name="ib_peskin", variant="srt_peskin", nx=64, ny=40, tau=0.6, pre_steps=30,
         n=32, radius=5.0, cx=12.3, cy=20.2),
]


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def sample_nodes(nx, ny, seed=7, n=48):
    """Boundary nodes of every kind plus seeded interior nodes, as (x, y)."""
    pts = {(0, 0), (0, ny - 1), (nx - 1, 0), (nx - 1, ny - 1), (0, ny // 2), (1, 1),
           (nx - 1, ny // 2), (nx - 2, ny - 2), (5, 0), (399, 0), (400, 0), (nx - 3, 0),
           (7, ny - 1), (nx // 2, 1), (nx // 2, ny - 2)}
    rng = np.random.default_rng(seed)
    while len(pts) < n:
        pts.add((int(rng.integers(0, nx)), int(rng.integers(0, ny))))
    return sorted(p for p in pts if 0 <= p[0] < nx and 0 <= p[1] < ny)


def export_nets(refroot):
    import torch

    out = os.path.join(HERE, "band_nets")
    os.makedirs(out, exist_ok=True)
    nets = {}
    for t in NET_TYPES:
        m = torch.jit.load(os.path.join(refroot, "NNmodel", f"AutoT0{t}.pt"), map_location="cpu")
        assert not m.training
        w = np.concatenate([p.detach().numpy().ravel() for _, p in m.named_parameters()])
        w = w.astype(np.float32)
        w.tofile(os.path.join(out, f"AutoT0{t}.f32"))
        nets[t] = (m, w)
    return nets


def net_golden(nets):
    import torch

    rng = np.random.default_rng(2024)
    res = {}
    for t, (m, _) in nets.items():
        n = 64
        ux = rng.uniform(-0.02, 0.14, size=(n, 5))
        uy = rng.uniform(-0.03, 0.03, size=(n, 5))
        rho = rng.uniform(0.97, 1.03, size=(n, 5))
        x = np.stack([ux, uy, rho], axis=2).reshape(n, 15).astype(np.float32)
        x[0] = np.array([0.1, 0.0, 1.0] * 5, np.float32)
        with torch.no_grad():
            y = m(torch.from_numpy(x)).numpy().reshape(-1)
            # batch-1 forwards, as the reference calls the net (mesh.cpp:2810-2819)
            y1 = np.array([m(torch.from_numpy(x[i:i + 1])).item() for i in range(n)], np.float32)
        res[f"x{t}"] = x
        res[f"y{t}"] = y1
        res[f"ybatch{t}"] = y
    np.savez(os.path.join(HERE, "band_net_golden.npz"), **res)
    return res


def plate_golden():
    import pyoracle as po

    nn_dir = os.path.join(HERE, "band_nets")
    cases = {}
    for c in PLATE_CASES:
        if c["nets"]:
            os.environ["IPPI_REF_NN_DIR"] = nn_dir
        else:
            os.environ.pop("IPPI_REF_NN_DIR", None)
        ref = po.RefSim(c["nx"], c["ny"], tau=c["tau"], cs=c["cs"], u_in=0.1,
                        avg_start=c["avg_start"], variant=c["variant"])
        pts = sample_nodes(c["nx"], c["ny"])
        snaps = []
        done = 0
        for s in c["steps"]:
            rc = ref.step(s - done, done + 1)
            done = s
            snap = {"step": s, "rc": rc, "hash": {}, "sample": {}}
            for fname, fid in (("F", po.F), ("rho", po.RHO), ("ux", po.UX), ("uy", po.UY),
                               ("avg_u", po.AVG_U), ("avg_v", po.AVG_V), ("avg_rho", po.AVG_RHO),
                               ("tau", po.TAU), ("nnflag", po.NNFLAG)):
                a = ref.get(fid)
                snap["hash"][fname] = sha(a)
                if fid == po.F:
                    snap["sample"][fname] = [[float(a[k, y, x]) for k in range(9)] for x, y in pts]
                else:
                    snap["sample"][fname] = [float(a[y, x]) for x, y in pts]
            snaps.append(snap)
        flags = ref.get(po.FLAGS).astype(np.uint8)
        cases[c["name"]] = dict(case=c, sample_nodes=pts, snapshots=snaps,
                                flags_sha=hashlib.sha256(flags.tobytes()).hexdigest(),
                                flags_rows=["".join(chr(v) for v in flags[y]) for y in
                                            (0, 1, c["ny"] - 1)])
        del ref
    os.environ.pop("IPPI_REF_NN_DIR", None)
    return cases


def ib_golden():
    import pyoracle as po

    cases = {}
    for c in IB_CASES:
        ref = po.RefSim(c["nx"], c["ny"], tau=c["tau"], u_in=0.1, variant=c["variant"])
        ref.step(c["pre_steps"], 1)
        pre = {f: ref.get(fid) for f, fid in (("ux", po.UX), ("uy", po.UY), ("rho", po.RHO))}
        xy, vref, mf, nf = ref.ib_probe(c["n"], c["radius"], c["cx"], c["cy"])
        ux_after = ref.get(po.UX)
        cases[c["name"]] = dict(
            case=c, pre_hash={k: sha(v) for k, v in pre.items()},
            xy=xy.tolist(), vref=vref.tolist(), mforce=mf.tolist(),
            nforce_hash=sha(nf), ux_after_hash=sha(ux_after),
            nforce_nonzero=[[int(y), int(x), float(nf[0, y, x]), float(nf[1, y, x])]
                            for y, x in zip(*np.nonzero(nf[0] != 0))])
        del ref
    return cases


def main():
    refroot = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IPPI_REFERENCE_DIR",
                                                                   "/root/reference")  # its mount point
    import pyoracle as po

    nets = export_nets(refroot)
    net_golden(nets)
    po.build_oracle()
    po.build_ref()
    golden = {"plate": plate_golden(), "ib": ib_golden()}
    with open(os.path.join(HERE, "ref_golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
