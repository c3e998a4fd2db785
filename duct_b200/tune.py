"""Offline tuner of the GEMM-pass kernels: times the library's pass-kernel
variants (tile shapes: 32 or 16 complex lines per CTA, the register-operand
and persistent forms, the flip-symmetric half-block passes) for a batch of
fields at each grid size and writes the fastest per size to a JSON table
keyed by (ny, nz).  `Context.apply_tuning()` reads the table back and sets
the pass kernel of the context's size class (ductgpu_set_pass_kernel) and,
for rectangular grids, the folded (one persistent launch, or one launch per
pass and half-block size) / full choice (ductgpu_set_rect_fold).

    python -m duct_b200.tune --square 33,65,129,193 --rect 65x129,49x145,33x129 \\
        --out duct_b200/tuning.json

Square grids: a substep's u, v, w (Dirichlet, lambda = kx^2 + 2/(nu dt))
and p (Neumann, lambda = kx^2) with `--modes` Fourier modes, every variant
timed over CUDA-graph replays.  Rectangular grids (my x mz, aspect mz/my):
the same four fields through ductgpu_solve_rect_fields_dev: folded, one
launch per pass and size, folded in one launch, and full operators.
Needs a GPU.
"""
import argparse
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

VARIANTS = {"staged-32": 0, "register": 1, "staged-16": 2, "persist": 3, "parity": 4, "parity-queue": 5}


def _time_graph(ctx, gid, reps):
    for _ in range(3):
        ctx.graph_launch(gid)
    ctx.synchronize()
    ctx.event_record(0)
    for _ in range(reps):
        ctx.graph_launch(gid)
    ctx.event_record(1)
    return ctx.event_elapsed(0, 1) / reps


def tune_square(ctx, m, nmodes, reps=20):
    import duct_b200 as D
    from duct_b200 import synth
    ctx.pseudomat(m)
    xalp = 0.5 * np.arange(nmodes)
    lam = 2.0 / ((1.0 / 2000.0) * 1.0e-3)
    fields, keep = [], []
    for k, (bound, lm) in enumerate((("d", lam), ("d", lam), ("d", lam), ("n", 0.0))):
        f = synth.chebyshev_rhs(m, m, nmodes, seed=1 + k, ib=0)
        r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
        r.upload(f)
        keep += [r, s]
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=lm, ib=0, bound=bound))
    ms = {}
    for name, v in VARIANTS.items():
        ctx.set_pass_kernel(v)
        try:
            gid = ctx.graph_create(fields)
        except D.DuctGPUError:
            continue
        ms[name] = _time_graph(ctx, gid, reps)
        ctx.graph_destroy(gid)
    ctx.set_pass_kernel(-1)
    for x in keep:
        x.free()
    best = min(ms, key=ms.get)
    return {"ny": m, "nz": m, "nmodes": nmodes, "fields": 4, "pass_kernel": best, "ms_per_batch": ms}


def tune_rect(ctx, my, mz, nmodes, reps=20):
    from duct_b200 import synth
    aspect = (mz - 1) / (my - 1)
    ctx.pseudomat_temp(0, my, mz, 1.0, aspect)
    ctx.pseudomat_temp(1, my, mz, 1.0, aspect, ("n", "n"), ("n", "n"))
    xalp = 1.0 * np.arange(nmodes)
    lam = 2.0 / ((1.0 / 4400.0) * 5.0e-4)
    fields, keep = [], []
    for k in range(4):
        neu = k == 3
        f = synth.chebyshev_rhs(my, mz, nmodes, seed=k, ib=0)
        r, s = ctx.device_array(f.shape), ctx.device_array(f.shape)
        r.upload(f)
        keep += [r, s]
        fields.append(dict(rhs=r, sol=s, xalp=xalp, alambda=0.0 if neu else lam, ib=0, slot=1 if neu else 0))
    ms = {}
    modes = {"full": 0, "fold": 1, "fold-one-launch": 2}
    for name, fold in modes.items():
        ctx.set_rect_fold(fold)
        gid = ctx.graph_create(fields, rect=True)
        ms[name] = _time_graph(ctx, gid, reps)
        ctx.graph_destroy(gid)
    ctx.set_rect_fold(1)
    for x in keep:
        x.free()
    return {"ny": my, "nz": mz, "nmodes": nmodes, "fields": 4, "rect_fold": modes[min(ms, key=ms.get)],
            "ms_per_batch": ms}


def apply(ctx, my, mz, path=TABLE):
    """Settings of the table entry for (my, mz) onto ctx; returns the entry
    (None if the table or the entry is missing: the library defaults stay)."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        table = json.load(f)
    for e in table.get("entries", []):
        if e["ny"] == my and e["nz"] == mz:
            if "pass_kernel" in e:
                n = my - 2
                size_class = 0 if n <= 63 else (1 if n <= 127 else 2)
                ctx.set_pass_kernel(VARIANTS[e["pass_kernel"]], size_class)
            if "rect_fold" in e:
                ctx.set_rect_fold(e["rect_fold"])
            return e
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--square", default="33,65,129,193")
    ap.add_argument("--rect", default="65x129,49x145,33x129")
    ap.add_argument("--modes", type=int, default=64)
    ap.add_argument("--out", default=TABLE)
    a = ap.parse_args()
    import duct_b200 as D
    entries = []
    with D.Context(0) as ctx:
        for s in filter(None, a.square.split(",")):
            entries.append(tune_square(ctx, int(s), a.modes))
            print(json.dumps(entries[-1]), flush=True)
        for s in filter(None, a.rect.split(",")):
            my, mz = (int(x) for x in s.split("x"))
            entries.append(tune_rect(ctx, my, mz, a.modes))
            print(json.dumps(entries[-1]), flush=True)
    import subprocess
    dev = subprocess.run(["nvidia-smi", "--query-gpu=name", "--format=csv,noheader"], capture_output=True,
                         text=True).stdout.strip().splitlines()
    with open(a.out, "w") as f:
        json.dump({"device": dev[0] if dev else None, "tuned_with": "python -m duct_b200.tune", "entries": entries},
                  f, indent=1)


if __name__ == "__main__":
    main()
