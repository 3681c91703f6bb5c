"""Project autotuner for the fast (mu nu|P) kernels.

Each (l_i, l_j | l_k) class has compiled variants that differ in the
accumulator budget per lane (how many warps split the ket components) and in
the register cap (how many warps stay resident per SM); see k3c_fast.cuh.
Which one wins depends on the class and the GPU, so the tuner times every
variant of every class on a real batch (each class kernel alone, CUDA events
on the batch's stream, best of a few launches) and keeps the fastest.  The
result is a small JSON cache (``tuning/b200_fp64.json``) that bench.py and
users load with :func:`apply`.
"""

import json
import pathlib

from ._lib import lib

N_VARIANTS = 6
DEFAULT_CACHE = pathlib.Path(__file__).resolve().parent / "tuning" / "b200_fp64.json"


def apply(table):
    """Set the library's variant for every class in {"li,lj,lk": variant}."""
    L = lib()
    for key, v in table.items():
        li, lj, lk = (int(x) for x in key.split(","))
        if L.eip_tune_set(li, lj, lk, int(v)) != 0:
            raise ValueError(f"invalid tuning entry {key}: {v}")


def load(path=DEFAULT_CACHE):
    p = pathlib.Path(path)
    if not p.exists():
        return None
    data = json.loads(p.read_text())
    apply(data["variants"])
    return data


def tune(batch, classes, repeats=3):
    """Time every variant of every class of `batch` (a ThreeCenterBatch with
    its output allocated) and set the fastest; returns (table, timings_ms)."""
    import torch

    L = lib()
    stream = torch.cuda.ExternalStream(batch.stream)
    table, timings = {}, {}
    for (li, lj, lk) in classes:
        if L.eip_tune_get(li, lj, lk) < 0:
            continue
        best = None
        for v in range(N_VARIANTS):
            L.eip_tune_set(li, lj, lk, v)
            if not batch.run_class(li, lj, lk):  # first launch also loads the module
                break
            times = []
            for _ in range(repeats):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                batch.run_class(li, lj, lk)
                e1.record(stream)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            t = min(times)
            timings[f"{li},{lj},{lk}:{v}"] = t
            if best is None or t < best[1]:
                best = (v, t)
        if best is not None:
            L.eip_tune_set(li, lj, lk, best[0])
            table[f"{li},{lj},{lk}"] = best[0]
    batch.status()
    return table, timings


def save(table, timings, meta, path=DEFAULT_CACHE):
    p = pathlib.Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    p.write_text(json.dumps({"variants": table, "timings_ms": timings, "meta": meta}, indent=1, sort_keys=True) + "\n")
