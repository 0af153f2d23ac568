"""Tile-width autotuner for the split-precision contractions, per (nao, naux).

The column tile of the tensor-core contraction kernel (gb200_set_tile_width) trades the width of
one MMA against tile-count rounding of each contraction's N (N = naux nao, naux, nk nao^2 or
ntau nao) and the per-tile epilogue work.  `measure` times the whole self-energy of a synthetic
system of the given (nao, naux) with every candidate width (CUDA events, after warm-up);
`tune` does so over a grid of shapes and `tile_table.json` next to this file holds the result of a
run on a B200 (python -m gb200.tune --out ...).  `choose_tile` reads the table: the entry of the
nearest measured shape (relative distance in nao and naux), 0 (the widest tile) without one.
"""
from __future__ import annotations

import argparse
import json
import math
import os

CANDIDATES = (32, 48, 64, 80, 96)
TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tile_table.json")


def load_table(path: str = TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f).get("shapes", {})


def choose_tile(nao: int, naux: int, table: dict | None = None) -> int:
    """Tile width for a system of (nao, naux) from the measured table (0: widest)."""
    table = load_table() if table is None else table
    best, dist = 0, math.inf
    for key, entry in table.items():
        a, q = (int(x) for x in key.split("x"))
        d = math.hypot(math.log(nao / a), math.log(naux / q))
        if d < dist:
            best, dist = int(entry["bn"]), d
    return best


def measure(nao: int, naux: int, slices: int = 5, nts: int = 80, mesh=(2, 2, 2), reps: int = 3,
            candidates=CANDIDATES, seed: int = 0, device: int = 0) -> dict:
    """Milliseconds of one split-precision self-energy of a synthetic system per tile width."""
    import torch

    from . import lib, solvers, synth

    s = synth.make_system(mesh=mesh, nao=nao, naux=naux, ns=1, beta=100.0, nts=nts, eps_range=2.0, seed=seed)
    ctx = solvers.make_context(s, device=device, precision=lib.PREC_SPLIT, slices=slices)
    try:
        G = torch.from_numpy(s.G).to(f"cuda:{device}")
        Sig = torch.empty_like(G)
        out = {}
        for bn in candidates:
            ctx.set_tile_width(bn)
            ctx.gw_sigma_device(G.data_ptr(), Sig.data_ptr())  # warm-up (buffers, maps)
            torch.cuda.synchronize(device)
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record()
            for _ in range(reps):
                ctx.gw_sigma_device(G.data_ptr(), Sig.data_ptr())
            ev[1].record()
            torch.cuda.synchronize(device)
            out[int(bn)] = ev[0].elapsed_time(ev[1]) / reps
        return out
    finally:
        ctx.close()


def tune(shapes, **kw) -> dict:
    """{"<nao>x<naux>": {"bn": fastest width, "ms": {width: ms}}} over `shapes` [(nao, naux)]."""
    table = {}
    for nao, naux in shapes:
        ms = measure(nao, naux, **kw)
        table[f"{nao}x{naux}"] = {"bn": min(ms, key=ms.get), "ms": ms}
    return table


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--slices", type=int, default=5)
    args = ap.parse_args(argv)
    shapes = [(nao, naux) for nao in (8, 16, 24, 32, 40, 48) for naux in (4 * nao, 6 * nao)]
    table = tune(shapes, slices=args.slices)
    import torch
    doc = {"device": torch.cuda.get_device_name(0), "slices": args.slices,
           "workload": "synthetic system per shape: 2x2x2 mesh, ntau = 80, beta = 100, one self-energy, "
                       "CUDA events over 3 calls after a warm-up call",
           "shapes": table}
    with open(args.out, "w") as f:
        json.dump(doc, f, indent=1)
    print(json.dumps({k: v["bn"] for k, v in table.items()}))


if __name__ == "__main__":
    main()
