"""Project autotuner for the fast (mu nu|P) kernels.

Each (l_i, l_j | l_k) class has compiled variants that differ in the
accumulator budget per lane (how many warps split the ket components) and in
the register cap (how many warps stay resident per SM); see k3c_fast.cuh.
Which one wins depends on the class and the GPU, so the tuner times every
variant of every class on a real batch (each class kernel alone, CUDA events
on the batch's stream, best of a few launches) and keeps the fastest.  The
result is a small JSON cache (``tuning/b200_fp64.json``) that bench.py and
users load with :func:`apply`.  The FP32 kernels of the mixed-precision path
have their own variants (0, 2, 3, 4), tuned on a batch whose every shell pair
takes the FP32 path (``variants_fp32`` in the cache).
"""

import json
import pathlib

from ._lib import lib

N_VARIANTS = 7
FP32_VARIANTS = (0, 2, 3, 4)
DEFAULT_CACHE = pathlib.Path(__file__).resolve().parent / "tuning" / "b200_fp64.json"


def apply(table, fp32=False):
    """Set the library's variant for every class in {"li,lj,lk": variant}."""
    L = lib()
    setter = L.eip_tune_set_fp32 if fp32 else L.eip_tune_set
    for key, v in table.items():
        li, lj, lk = (int(x) for x in key.split(","))
        if setter(li, lj, lk, int(v)) != 0:
            raise ValueError(f"invalid tuning entry {key}: {v}")


def load(path=DEFAULT_CACHE):
    p = pathlib.Path(path)
    if not p.exists():
        return None
    data = json.loads(p.read_text())
    apply(data["variants"])
    if "variants_fp32" in data:
        apply(data["variants_fp32"], fp32=True)
    return data


def tune(batch, classes, repeats=3, fp32=False):
    """Time every variant of every class of `batch` (a ThreeCenterBatch with
    its output allocated) and set the fastest; returns (table, timings_ms).
    fp32: tune the FP32 kernels (give a mixed batch whose pairs all take FP32)."""
    import torch

    L = lib()
    get = L.eip_tune_get_fp32 if fp32 else L.eip_tune_get
    set_ = L.eip_tune_set_fp32 if fp32 else L.eip_tune_set
    variants = FP32_VARIANTS if fp32 else range(N_VARIANTS)
    stream = torch.cuda.ExternalStream(batch.stream)
    table, timings = {}, {}
    for (li, lj, lk) in classes:
        if get(li, lj, lk) < 0:
            continue
        best = None
        for v in variants:
            set_(li, lj, lk, v)
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
            set_(li, lj, lk, best[0])
            table[f"{li},{lj},{lk}"] = best[0]
    batch.status()
    return table, timings


def save(table, timings, meta, path=DEFAULT_CACHE, table_fp32=None, timings_fp32=None):
    p = pathlib.Path(path)
    p.parent.mkdir(parents=True, exist_ok=True)
    data = {"variants": table, "timings_ms": timings, "meta": meta}
    if table_fp32 is not None:
        data["variants_fp32"] = table_fp32
        data["timings_fp32_ms"] = timings_fp32
    p.write_text(json.dumps(data, indent=1, sort_keys=True) + "\n")
