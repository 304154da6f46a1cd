"""Tune the tile configuration (sweeps per step S, tile height) of the red-black
SOR solve for this GPU with ``pt_autotune``, on the shapes of the workloads it
serves, and write the table the library reads.

    python -m paintop_b200.tune [--workloads screened_2048,batch_uneven,multi_4096]
                                [--repeats 3] [--table FILE] [--write-inc]

For each workload the whole call is timed under every configuration (device
buffers, CUDA events on the context's stream, best of ``repeats``), and the
fastest goes into the shape-keyed table. An entry already in the table is kept
unless a new configuration beats it by more than 5 %, so re-tuning does not
flip near-equal choices. ``--table`` names the table file (one ``key config``
pair per line; the library reads it from ``$PAINTOP_CUDA_TUNE_TABLE``).
``--write-inc`` also rewrites ``csrc/tune_table_b200.inc``, the entries compiled
into the library, with each workload's timings as comments.

Workloads (the benchmark's seeded generators, ``paintop_b200.synth``):
  screened_2048  2048x2048 RGBA, lambda 0.01, star mask, rel-res 1e-6, omega 1.8
  batch_uneven   256 RGB instances of uneven sizes, rel-res 1e-6, automatic omega
  multi_4096     4096x4096 RGB, 8 polygons, lambda 0, rel-res 1e-6, automatic omega
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(HERE, "csrc", "tune_table_b200.inc")
WORKLOADS = ("screened_2048", "batch_uneven", "multi_4096")


def shape_key(problems) -> int:
    """The library's table key (autotune.cpp, shape_key): floor(log2) of the
    total pixel count over all channels, floor(log2) of the largest image,
    whether lambda is zero for all problems, whether the call holds a batch."""
    total, largest, lam0 = 0.0, 1.0, True
    for p in problems:
        px = float(p["width"]) * p["height"]
        total += px * p["channels"]
        largest = max(largest, px)
        lam0 = lam0 and p["lam"] == 0.0
    lt = max(0, math.floor(math.log2(max(total, 1.0))))
    ll = max(0, math.floor(math.log2(largest)))
    return (lt << 16) | (ll << 8) | (2 if lam0 else 0) | (1 if len(problems) > 1 else 0)


def workload_problems(name: str):
    """(problem dicts, flags) of a workload, images as host arrays."""
    from paintop_b200 import _lib, synth
    if name == "screened_2048":
        insts, lam, flags, omega = [synth.screened_2048(1)], 0.01, 0, 1.8
    elif name == "batch_uneven":
        insts, lam, flags, omega = synth.batch_uneven(1, 256), 0.0, _lib.PT_FLAG_OMEGA_AUTO, 1.8
    elif name == "multi_4096":
        insts, lam, flags, omega = [synth.multi_4096(1)], 0.0, _lib.PT_FLAG_OMEGA_AUTO, 1.8
    else:
        raise ValueError(f"unknown workload {name!r}")
    max_it = 2000 if name == "screened_2048" else 100000
    probs = [dict(width=i.width, height=i.height, channels=i.channels, source=i.source, target=i.target,
                  mask=i.mask, lam=lam, max_iterations=max_it, tolerance=1e-6, omega=omega, flags=flags)
             for i in insts]
    return probs


def autotune(ctx, probs, repeats: int = 3):
    """pt_autotune over device copies of `probs` -> (chosen config, ms per config)."""
    import torch
    from paintop_b200 import _lib
    dev = torch.device("cuda", ctx.device)
    n = len(probs)
    keep = []
    arr = (_lib.PtProblem * n)()
    outs = (C.c_void_p * n)()
    reps = [(_lib.PtReport * (p["channels"] + 1))() for p in probs]
    rep_ptrs = (C.POINTER(_lib.PtReport) * n)(*[C.cast(r, C.POINTER(_lib.PtReport)) for r in reps])
    for k, p in enumerate(probs):
        s = torch.as_tensor(p["source"].reshape(-1), device=dev)
        t = torch.as_tensor(p["target"].reshape(-1), device=dev)
        m = torch.as_tensor(p["mask"].reshape(-1), device=dev)
        o = torch.empty_like(s)
        keep += [s, t, m, o]
        arr[k] = _lib.PtProblem(p["width"], p["height"], p["channels"], s.data_ptr(), t.data_ptr(),
                                m.data_ptr(), p["lam"], p["max_iterations"], p["tolerance"], p["omega"],
                                p["flags"] | _lib.PT_FLAG_DEVICE_POINTERS, None)
        outs[k] = o.data_ptr()
    torch.cuda.synchronize(dev)
    ncfg = int(_lib.lib().pt_tile_config_count())
    ms = (C.c_double * ncfg)()
    chosen = C.c_int32(-1)
    st = _lib.lib().pt_autotune(ctx.h, arr, n, int(repeats), outs, rep_ptrs, C.byref(chosen), ms)
    if st != _lib.PT_OK:
        raise _lib.CudaError(st, ctx.last_error())
    converged = all(r[c].converged for r, p in zip(reps, probs) for c in range(p["channels"]))
    return int(chosen.value), [float(x) for x in ms], converged, keep


def config_label(cfg: int) -> str:
    from paintop_b200 import _lib
    s, w, h = C.c_int32(), C.c_int32(), C.c_int32()
    _lib.lib().pt_tile_config_info(cfg, C.byref(s), C.byref(w), C.byref(h))
    return f"S={s.value} tile {w.value}x{h.value}"


def write_inc(entries: list[dict], path: str = INC) -> None:
    lines = ["// B200 tile-configuration table: {shape key, configuration}. Written by",
             "// `python -m paintop_b200.tune --write-inc` (pt_autotune, device buffers, best",
             "// of the given repeats per configuration); ms per configuration in the comments."]
    for e in sorted(entries, key=lambda e: e["key"]):
        times = ", ".join(f"{t:.2f}" for t in e["ms_per_config"])
        lines.append(f"// {e['workload']}: {config_label(e['config'])}; ms per config [{times}]")
        lines.append(f"{{0x{e['key']:08x}u, {e['config']}}},")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workloads", default=",".join(WORKLOADS))
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--table", default=None, help="table file to write (PAINTOP_CUDA_TUNE_TABLE)")
    ap.add_argument("--write-inc", action="store_true")
    ap.add_argument("--json", default=None, help="write the measurements here")
    ap.add_argument("--from-json", default=None,
                    help="write the .inc from measurements saved by --json (no GPU needed)")
    args = ap.parse_args(argv)
    if args.from_json:
        with open(args.from_json) as f:
            write_inc(json.load(f))
        return 0
    if args.table:
        os.environ["PAINTOP_CUDA_TUNE_TABLE"] = os.path.abspath(args.table)
    import torch
    torch.cuda.set_device(0)
    from paintop_b200 import _lib
    ctx = _lib.Context(0)
    entries = []
    try:
        for name in args.workloads.split(","):
            probs = workload_problems(name)
            cfg, ms, conv, _ = autotune(ctx, probs, args.repeats)
            e = dict(workload=name, key=shape_key(probs), config=cfg, ms_per_config=ms, converged=conv,
                     fastest=int(min(range(len(ms)), key=lambda k: ms[k])))
            entries.append(e)
            print(json.dumps(e), flush=True)
    finally:
        ctx.close()
    if args.write_inc:
        write_inc(entries)
    if args.json:
        with open(args.json, "w") as f:
            json.dump(entries, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
