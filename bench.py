#!/usr/bin/env python
"""Benchmark: screened (mu nu|P) triplets/s on the batched B200 path.

Workload (one "step"): every (mu nu|P) integral of 64 seeded synthetic organic
molecules of 3-60 atoms (log-uniform; H/C/N/O 0.5/0.3/0.1/0.1; bonded growth;
orbital 3s2p1d / H 2s1p contracted, auxiliary uncontracted s-g), computed as
one CUDA-graph launch of the batched library path into a packed device
buffer.  Metric unit: contracted shell triplets with Schwarz-type bound
>= 1e-14 per second (all of them are computed).

  value   device-resident tables, K graph launches timed with CUDA events on
          the library's stream;
  e2e     through the C ABI each step: H2D copy of every input table from the
          batch's pinned host copy and of the 64 molecules' densities, the
          graph, the density-fitted Coulomb matrix of every molecule (the
          library's gamma and J kernels over the packed output, Cholesky
          solves with factors made once per geometry), and a D2H copy of the
          64 J matrices;
  roofline  the class kernel with the largest device time, run alone,
          algorithmic FLOPs (roofline.py) / its CUDA-event time, against the
          FP64 FMA peak measured on the same GPU by the library's
          microbenchmark;
  cpu_baseline  the reference library (oracle/_ref, its own C++/OpenMP path)
          on a bounded sample of the same molecules, all host cores.

Also in the line (not part of the timed step): `cpu_baseline.gpu_same_sample`,
the batched GPU path on exactly the CPU sample's molecules; `dropin_fp64`, the
plain FP64 drop-in three_center on that sample; `serving`, Poisson streams of
5-200-atom requests (S, V, (P|Q), (mu nu|P)) at several rates through the
continuous-batching server, p50/p99 latency, beside the same requests served
alone in FP64; `water100_mixed_vs_fp64`, the 100-water cluster's (mu nu|P) in
FP64 and mixed precision window by window, max abs/rel error per class and
triplets/s of both; `water10_per_type`, the 10-water S, V, (P|Q), (mu nu|P)
through the drop-in beside the reference library at all host threads and 1
thread; `random_triplets_high_l`, 2000 random shell triplets up to (g g|h) in
FP64 and mixed precision against the reference library; `mixed_vs_reference`,
the mixed path's error against the reference library per integral type and
class.

`--impl reference` times only that reference path (per step: the sample) and
prints its own line.  Under torchrun each rank runs its own 64 molecules
(seed + rank): independent shards, no data-path collective (weak scaling).
"""

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

REPO = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "screened (μν|P) triplets/s, mixed vs FP64 at ≤1e-10 abs; p50/p99 latency"
UNIT = "triplets/s"
WORKLOAD = ("batched uneven sizes: 64 organic molecules of 3-60 atoms (log-uniform, H/C/N/O), "
            "orbital 3s2p1d/2s1p contracted, auxiliary s-g uncontracted, all (mu nu|P) spherical, "
            "one CUDA-graph launch")
THRESHOLD = 1e-14


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def shard_seed(seed, rank):
    """Each rank's molecules: an independent shard of the same generator."""
    return seed + 1000 * rank


def reduce_over_ranks(values, op, device):
    """All-reduce a list of floats over the process group (identity when alone)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return t.tolist()


def build_workload(seed, n_mol):
    import importlib

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    mols = syn.organic_batch(seed, n_mol)
    pds = [pu.form_pair_data(m, 1e-14) for m in mols]
    ads = [pu.form_auxiliary_pair_data(m) for m in mols]
    stats = [rf.class_statistics(pd, ad, THRESHOLD) for pd, ad in zip(pds, ads)]
    return mols, pds, ads, stats


def reference_sample(mols, pds, ads, stats, budget_s, max_dense=2.0e8):
    """Time the reference library on molecules (in batch order, skipping any whose
    dense output exceeds max_dense doubles) until budget_s seconds elapse."""
    import numpy as np
    import oracle

    ref = oracle.reference()
    if ref is None:
        return None
    done, triplets, t_total = [], 0, 0.0
    for i, m in enumerate(mols):
        if m.n_aux * m.n_ao * m.n_ao > max_dense:
            continue
        t0 = time.perf_counter()
        oracle.drive_three_center(ref, pds[i], ads[i], m)
        t_total += time.perf_counter() - t0
        triplets += sum(d["screened"] for d in stats[i].values())
        done.append(i)
        if t_total >= budget_s:
            break
    return dict(value=triplets / t_total, seconds=t_total, molecules=done, triplets=triplets,
                cores=os.cpu_count())


class ClockSampler:
    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.f.close()

    def summary(self, device_index):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines()]
        except Exception:
            return None
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9 and r[0].strip() == str(device_index)]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows)}


def mixed_error(bt, mols, pds, ads, threshold, torch, budget_bytes=30e9):
    """Max |mixed - FP64| over the packed (mu nu|P) of the leading molecules whose
    output fits budget_bytes (both results resident at once)."""
    take, total = [], 0
    for i, m in enumerate(mols):
        b = 8 * m.n_ao * m.n_ao * m.n_aux  # dense size; the packed output is about half
        if total + b > 2 * budget_bytes:
            break
        take.append(i)
        total += b
    sub = [mols[i] for i in take], [pds[i] for i in take], [ads[i] for i in take]
    f64 = bt.ThreeCenterBatch(*sub, precision="fp64")
    mix = bt.ThreeCenterBatch(*sub, precision="mixed", fp32_threshold=threshold)
    n = f64.output_elems
    a = torch.empty(n, dtype=torch.float64, device="cuda")
    c = torch.empty(n, dtype=torch.float64, device="cuda")
    f64.bind_output(a.data_ptr())
    mix.bind_output(c.data_ptr())
    f64.run()
    mix.run()
    f64.status()
    mix.status()
    d = (a - c).abs()
    big = a.abs() > 1e-6
    rel = float(((a - c).abs() / a.abs().clamp_min(1e-300))[big].max()) if bool(big.any()) else 0.0
    out = {"max_abs": float(d.max()), "max_rel_where_abs_gt_1e-6": rel, "molecules": len(take),
           "elements": n}
    f64.bind_output(0)
    mix.bind_output(0)
    f64.close()
    mix.close()
    del a, c
    torch.cuda.empty_cache()
    return out


def same_sample_rate(bt, torch, mols, pds, ads, smp, args):
    """The batched GPU path (FP64 and mixed) on exactly the cpu_baseline's
    molecules, CUDA events: screened triplets/s like for like."""
    idx = smp["molecules"]
    out = {}
    for prec in ("fp64", "mixed"):
        b = bt.ThreeCenterBatch([mols[i] for i in idx], [pds[i] for i in idx], [ads[i] for i in idx],
                                precision=prec, fp32_threshold=args.fp32_threshold)
        b.alloc_output()
        st = torch.cuda.ExternalStream(b.stream)
        for _ in range(args.warmup):
            b.run(sync=False)
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            b.run(sync=False)
        e1.record(st)
        b.sync()
        b.status()
        ms = e0.elapsed_time(e1) / args.steps
        out[prec] = {"ms_per_step": ms, "value": smp["triplets"] / (ms * 1e-3)}
        b.close()
    torch.cuda.empty_cache()
    out["ratio_mixed_vs_cpu"] = out["mixed"]["value"] / smp["value"]
    return out


def dropin_sample(mols, pds, ads, stats, sample_idx):
    """The plain FP64 drop-in three_center (reference C ABI, host buffers, dense
    output) on the GPU over the cpu_baseline's sample molecules."""
    import importlib

    mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
    if not sample_idx:
        return None
    mi.three_center(pds[sample_idx[0]], ads[sample_idx[0]], mols[sample_idx[0]])  # warm-up
    t0 = time.perf_counter()
    triplets = 0
    for i in sample_idx:
        mi.three_center(pds[i], ads[i], mols[i])
        triplets += sum(d["screened"] for d in stats[i].values())
    dt = time.perf_counter() - t0
    return {"value": triplets / dt, "unit": UNIT, "seconds": dt, "molecules": list(sample_idx),
            "what": "drop-in three_center per class, FP64, dense host output (wall clock incl. copies)"}


def run_serving(args, torch, seed):
    """Open-loop Poisson streams of requests (S, V, (P|Q), (mu nu|P)) of 5-200-atom
    molecules (the first `serve_requests` of the seeded 10k-request stream)
    through the continuous-batching server (mixed precision) at each rate of
    `serve_rates` (below, near and above the server's capacity), and the first
    `serve_alone` requests each served alone in FP64 with nothing else in flight."""
    import importlib

    import numpy as np

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    sv = importlib.import_module("electron-integral-playground_b200.serving")
    n = args.serve_requests
    sizes = syn.molecule_sizes(n, 5, 200, seed + 7)
    # requests carry only the molecule: the server builds its pair tables on
    # the device (and the auxiliary tables) after arrival, inside the latency
    mols = [syn.attach_synthetic_basis(syn.organic_molecule(na, seed * 7919 + i), aux_l_max=4, seed=seed)
            for i, na in enumerate(sizes)]
    free, _ = torch.cuda.mem_get_info()
    budget = min(150e9, free - 12e9)
    server = sv.IntegralServer(budget_bytes=budget, precision="mixed", fp32_threshold=args.fp32_threshold)
    server.serve([sv.Request(-1, mols[0], arrival=0.0)], realtime=False)  # warm-up
    rates = [float(r) for r in args.serve_rates.split(",") if r.strip()]
    per_rate = []
    pieces = None
    for k, rate in enumerate(rates):
        arrivals = np.cumsum(np.random.default_rng(seed + 11 + k).exponential(1.0 / rate, n))
        reqs = [sv.Request(i, m, arrival=float(t)) for i, (m, t) in enumerate(zip(mols, arrivals))]
        server.launches = 0
        server.host_s = {key: 0.0 for key in server.host_s}
        st = server.serve(reqs, realtime=True)
        if pieces is None:
            pieces = sum(len(server.pieces_of(r)) for r in reqs)
        per_rate.append({"rate_rps": rate, "requests": n, "throughput_rps": st["throughput_rps"],
                         "wall_s": st["wall_s"], "latency_p50_ms": st["latency_p50_s"] * 1e3,
                         "latency_p99_ms": st["latency_p99_s"] * 1e3,
                         "latency_p50_ci_ms": [x * 1e3 for x in st["latency_p50_ci_s"]],
                         "latency_p99_ci_ms": [x * 1e3 for x in st["latency_p99_ci_s"]], "launches": st["launches"],
                         "host_s": st["host_s"]})
    del server
    torch.cuda.empty_cache()
    alone = []
    # the same work per request as served (S included), nothing else in flight
    solo = sv.IntegralServer(budget_bytes=budget, precision="fp64", max_inflight=1)
    for i, m in enumerate(mols[:args.serve_alone]):
        alone.append(solo.serve([sv.Request(i, m, arrival=0.0)], realtime=False)["latency_p50_s"])
    del solo
    torch.cuda.empty_cache()
    lat_alone = np.array(alone)
    return {
        "requests": n, "atoms": [int(x) for x in sizes], "budget_gb": budget / 1e9, "precision": "mixed",
        "pieces": pieces, "rates": per_rate,
        "alone_fp64": {"requests": len(alone), "sum_s": float(lat_alone.sum()),
                       "throughput_rps": len(alone) / float(lat_alone.sum()),
                       "latency_p50_ms": float(np.percentile(lat_alone, 50)) * 1e3,
                       "latency_p99_ms": float(np.percentile(lat_alone, 99)) * 1e3,
                       "note": "each request served alone (nothing else in flight), FP64, same work "
                               f"(S, V, (P|Q), (mu nu|P)); first {len(alone)} requests"},
        "sample": f"the first {n} requests of the seeded 10k-request stream (5-200 atoms log-uniform), "
                  f"Poisson arrivals at each rate; requests carry molecules, pair tables are built on the "
                  f"device after arrival",
    }


def run_water100_windows(torch, bt, threshold, seed=0, window_bytes=24e9):
    """100-water cluster (300 atoms, 15 A cube, aux s-f): every (mu nu|P) in
    FP64 and in mixed precision, window by window over the auxiliary basis on
    resident tables; max abs / rel error of mixed vs FP64 per class, triplets/s
    of both (screen 1e-12), and the FP64 (P|Q) metric."""
    import importlib

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    sv = importlib.import_module("electron-integral-playground_b200.serving")
    mol = syn.water100_cluster(seed)
    pd, ad = pu.form_pair_data(mol, 1e-14), pu.form_auxiliary_pair_data(mol)
    stats = rf.class_statistics(pd, ad, 1e-12)
    screened = sum(v["screened"] for v in stats.values())
    b64 = bt.ThreeCenterBatch([mol], [pd], [ad], precision="fp64")
    bmx = bt.ThreeCenterBatch([mol], [pd], [ad], precision="mixed", fp32_threshold=threshold)
    full = b64.window()
    width = max(1, int(mol.n_aux * (window_bytes / 8) / full))
    edges = sv.window_edges(ad, mol.n_aux, width)
    sizes = [b64.window([lo], [hi]) for lo, hi in zip(edges[:-1], edges[1:])]
    buf_a = torch.empty(max(sizes), dtype=torch.float64, device="cuda")
    buf_b = torch.empty(max(sizes), dtype=torch.float64, device="cuda")
    classes = [(li, lj, lk) for (li, lj) in pd for lk in ad]
    err = {c: [0.0, 0.0] for c in classes}
    ms = {"fp64": 0.0, "mixed": 0.0}
    for lo, hi in zip(edges[:-1], edges[1:]):
        for name, b, buf in (("fp64", b64, buf_a), ("mixed", bmx, buf_b)):
            b.window([lo], [hi])
            st = torch.cuda.ExternalStream(b.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.run_window(buf.data_ptr())
            e1.record(st)
            b.sync()
            ms[name] += e0.elapsed_time(e1)
        for c in classes:
            ba, bb = b64.window_block(0, *c), bmx.window_block(0, *c)
            if ba is None or ba[2] == 0:
                continue
            n = ba[1] * (2 * c[0] + 1) * (2 * c[1] + 1) * (2 * c[2] + 1) * ba[2]
            x, y = buf_a[ba[0]:ba[0] + n], buf_b[bb[0]:bb[0] + n]
            d = (x - y).abs()
            big = x.abs() > 1e-6
            err[c][0] = max(err[c][0], float(d.max()))
            if bool(big.any()):
                err[c][1] = max(err[c][1], float((d[big] / x[big].abs()).max()))
    b64.status()
    bmx.status()
    split = {c: bmx.precision_split(*c) for c in classes}
    b64.close()
    bmx.close()
    del buf_a, buf_b
    torch.cuda.empty_cache()
    # (P|Q): FP64 (it feeds a Cholesky), one-centre pair classes on the same kernels
    bm = bt.ThreeCenterBatch([mol], [bt.metric_pair_tables(ad)], [ad], precision="mixed")
    bm.alloc_output()
    bm.run()
    st = torch.cuda.ExternalStream(bm.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    bm.run()
    e1.record(st)
    bm.sync()
    bm.status()
    pq_ms = e0.elapsed_time(e1)
    pq_bytes = bm.output_bytes
    bm.close()
    torch.cuda.empty_cache()
    n32 = sum(v[1] for v in split.values() if v)
    n64 = sum(v[0] for v in split.values() if v)
    return {
        "workload": "100 waters in a 15 A cube (300 atoms), orbital O 3s2p1d / H 2s1p, aux s-f; "
                    f"n_ao {mol.n_ao}, n_aux {mol.n_aux}",
        "packed_output_bytes": 8 * full, "windows": len(sizes), "screened_triplets_1e-12": screened,
        "fp64": {"ms": ms["fp64"], "triplets_per_s": screened / (ms["fp64"] * 1e-3)},
        "mixed": {"ms": ms["mixed"], "triplets_per_s": screened / (ms["mixed"] * 1e-3),
                  "fp32_threshold": threshold, "fp32_fraction_of_triplets": n32 / max(1, n32 + n64)},
        "mixed_vs_fp64_by_class": {f"{c[0]}{c[1]}|{c[2]}": {"max_abs": e[0], "max_rel_where_abs_gt_1e-6": e[1],
                                                             "fp32_triplets": split[c][1] if split[c] else 0}
                                   for c, e in sorted(err.items())},
        "max_abs_all_classes": max(e[0] for e in err.values()),
        "metric_PQ": {"precision": "fp64 (one-centre pairs never take the FP32 path)", "ms": pq_ms,
                      "bytes": pq_bytes},
    }


def best_of(fn, repeats=3):
    """(best wall seconds of `repeats` calls after one warm-up call, last result)."""
    out = fn()
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        out = fn()
        best = min(best, time.perf_counter() - t0)
    return best, out


def aux_slice(aux_data, n_aux, frac):
    """The auxiliary primitives of the shells whose first function lies in the
    first `frac` of the auxiliary functions (same n_aux: a slice of the output)."""
    from copy import copy

    import numpy as np

    out = {}
    for lk, a in aux_data.items():
        keep = np.asarray(a.i_ao_start) < frac * n_aux
        if keep.any():
            b = copy(a)
            b.A_a = np.ascontiguousarray(a.A_a[keep])
            b.coefficient = np.ascontiguousarray(np.asarray(a.coefficient)[keep])
            b.i_ao_start = np.ascontiguousarray(np.asarray(a.i_ao_start)[keep])
            out[lk] = b
    return out


def run_water10_per_type(seed=0):
    """10-water cluster (30 atoms), O 3s2p1d / H 2s1p, aux s-f, spherical: S, V,
    (P|Q) and (mu nu|P) through the drop-in C ABI (host arrays in and out, the
    reference front end's per-class calls), each timed as best of 3 after a
    warm-up; the reference library (oracle/_ref) on the same inputs with all
    host threads and with 1 thread ((mu nu|P) at 1 thread on the first eighth
    of the auxiliary functions); max |GPU - reference| per type."""
    import importlib

    import numpy as np

    import oracle

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    pu = importlib.import_module("electron-integral-playground_b200.pair_utility")
    mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    mol = syn.water10_cluster(seed)
    pd, ad = pu.form_pair_data(mol, 1e-14), pu.form_auxiliary_pair_data(mol)
    charges = np.asarray(mol.geometry, dtype=np.float64)
    tot, _ = rf.totals([rf.class_statistics(pd, ad, THRESHOLD)])
    gpu = {"S": lambda: mi.overlap(pd, mol), "V": lambda: mi.nuclear_attraction(pd, mol, charges),
           "PQ": lambda: mi.two_center(ad, mol), "3c": lambda: mi.three_center(pd, ad, mol)}
    out = {"workload": "10 waters in a 9 A cube (30 atoms), orbital O 3s2p1d / H 2s1p contracted, aux s-f, "
                       f"spherical; n_ao {mol.n_ao}, n_aux {mol.n_aux}",
           "primitive_pairs": int(sum(p.P_p.shape[0] for p in pd.values())),
           "aux_primitives": int(sum(a.A_a.shape[0] for a in ad.values())),
           "primitive_triplets_3c": int(tot["primitive"]), "screened_triplets_3c": int(tot["screened"]),
           "what": "wall time per integral type through the drop-in entry points (H2D, kernels, D2H, host "
                   "scatter into the dense reference layout); best of 3 after one warm-up", "types": {}}
    res = {}
    for k, f in gpu.items():
        t, v = best_of(f)
        res[k] = v
        out["types"][k] = {"gpu_ms": t * 1e3}
    ref = oracle.reference()
    if ref is None:
        out["reference"] = "reference library not built (make -C oracle ref)"
        return out
    nproc = os.cpu_count() or 1
    refs = {"S": lambda: oracle.drive_overlap(ref, pd, mol),
            "V": lambda: oracle.drive_nuclear_attraction(ref, pd, mol, charges),
            "PQ": lambda: oracle.drive_two_center(ref, ad, mol),
            "3c": lambda: oracle.drive_three_center(ref, pd, ad, mol)}
    oracle.set_reference_threads(nproc)
    for k, f in refs.items():
        t, v = best_of(f, 2)
        d = out["types"][k]
        d["reference_ms_all_threads"] = t * 1e3
        d["max_abs_gpu_vs_reference"] = float(np.max(np.abs(res[k] - v)))
        d["gpu_speedup_vs_all_threads"] = t * 1e3 / d["gpu_ms"]
    res = None
    oracle.set_reference_threads(1)
    for k in ("S", "V", "PQ"):
        t, _ = best_of(refs[k], 1)
        out["types"][k]["reference_ms_1_thread"] = t * 1e3
    sl = aux_slice(ad, mol.n_aux, 0.125)
    sl_tot, _ = rf.totals([rf.class_statistics(pd, sl, THRESHOLD)])
    t, _ = best_of(lambda: oracle.drive_three_center(ref, pd, sl, mol), 1)
    oracle.set_reference_threads(nproc)
    t_full = out["types"]["3c"]["reference_ms_all_threads"] * 1e-3
    out["types"]["3c"].update({
        "reference_1_thread_slice": {"ms": t * 1e3, "primitive_triplets": int(sl_tot["primitive"]),
                                     "what": "first eighth of the auxiliary functions, 1 thread"},
        "reference_1_thread_primitive_triplets_per_s": sl_tot["primitive"] / t,
        "reference_all_threads_primitive_triplets_per_s": tot["primitive"] / t_full,
        "gpu_primitive_triplets_per_s": tot["primitive"] / (out["types"]["3c"]["gpu_ms"] * 1e-3),
        "gpu_screened_triplets_per_s": tot["screened"] / (out["types"]["3c"]["gpu_ms"] * 1e-3)})
    out["reference"] = {"kind": "reference", "threads_all": nproc, "cpu_model": oracle.cpu_model()}
    return out


def run_random_high_l_triplets(torch, bt, fp64_peak, steps=5, seed=0, reference=True):
    """2000 random shell triplets (orbital l <= 4, aux l <= 5, 1-8 primitives,
    exponents log-uniform in [0.05, 1e4], centres in a 6 A cube), each its own
    molecule slot of one batch: FP64 and mixed precision, one CUDA-graph launch
    per step timed with CUDA events; triplets/s, integrals/s, the step's
    algorithmic FP64 rate; both against the reference library per triplet
    (max |error| per class, scaled by max(1, max|reference|)) and the reference
    library's own time for the 2000 calls (all host threads and 1 thread)."""
    import importlib

    import numpy as np

    import oracle

    syn = importlib.import_module("electron-integral-playground_b200.synthetic")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    lm = importlib.import_module("electron-integral-playground_b200._lib")
    trip = syn.random_shell_triplets(seed, 2000)
    mols = [t[4] for t in trip]
    pds = [{t[0]: t[1]} for t in trip]
    ads = [{t[2]: t[3]} for t in trip]
    flops = sum(t[1].P_p.shape[0] * t[3].A_a.shape[0] * rf.flops_per_primitive_triplet(t[0][0], t[0][1], t[2])
                for t in trip)
    out = {"workload": "2000 random shell triplets: orbital l <= 4 (g), auxiliary l <= 5 (h), 1-8 primitives, "
                       "exponents log-uniform in [0.05, 1e4], centres in a 6 A cube; one molecule slot each",
           "triplets": 2000, "algorithmic_flops_per_step": flops}
    dense = {}
    for prec in ("fp64", "mixed"):
        b = bt.ThreeCenterBatch(mols, pds, ads, precision=prec)
        b.alloc_output()
        st = torch.cuda.ExternalStream(b.stream)
        for _ in range(3):
            b.run(sync=False)
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            b.run(sync=False)
        e1.record(st)
        b.sync()
        b.status()
        ms = e0.elapsed_time(e1) / steps
        out[prec] = {"ms_per_step": ms, "triplets_per_s": 2000 / (ms * 1e-3),
                     "integrals_per_s": b.output_elems / (ms * 1e-3), "launches_per_step": b.launches_per_run}
        if prec == "fp64":
            out[prec]["achieved_tflops"] = flops / (ms * 1e-3) / 1e12
            out[prec]["frac_of_fp64_peak"] = flops / (ms * 1e-3) / 1e12 / fp64_peak
        buf = np.empty(b.output_elems)
        b._check(b.L.eip_batch_copy_output(b.h, 0, b.output_elems, lm.dp(buf)), "copy")
        dense[prec] = (b, buf)
    ref = oracle.reference() if reference else None
    f64, mix = dense["fp64"][0], dense["mixed"][0]
    out["mixed_vs_fp64_max_abs"] = float(np.max(np.abs(dense["fp64"][1] - dense["mixed"][1])))
    if ref is not None:
        nproc = os.cpu_count() or 1
        per_class = {}
        t_all, above = 0.0, []
        oracle.set_reference_threads(nproc)
        for m, (lij, pair, lk, aux, mol) in enumerate(trip):
            t0 = time.perf_counter()
            want = oracle.drive_three_center(ref, {lij: pair}, {lk: aux}, mol)
            t_all += time.perf_counter() - t0
            scale = max(1.0, float(np.max(np.abs(want))))
            e64 = float(np.max(np.abs(f64.dense(m) - want))) / scale
            emx = float(np.max(np.abs(mix.dense(m) - want))) / scale
            key = f"{lij[0]}{lij[1]}|{lk}"
            if e64 > 1e-12:
                above.append(m)
            c = per_class.setdefault(key, [0, 0.0, 0.0])
            c[0] += 1
            c[1] = max(c[1], e64)
            c[2] = max(c[2], emx)
        oracle.set_reference_threads(1)
        t0 = time.perf_counter()
        for (lij, pair, lk, aux, mol) in trip[:200]:
            oracle.drive_three_center(ref, {lij: pair}, {lk: aux}, mol)
        t_one = (time.perf_counter() - t0) * 10
        oracle.set_reference_threads(nproc)
        out["vs_reference"] = {
            "what": "max over the class's triplets of max|GPU - reference| / max(1, max|reference|)",
            "fp64_worst": max(v[1] for v in per_class.values()), "mixed_worst": max(v[2] for v in per_class.values()),
            "fp64_triplets_above_1e-12": above,
            "by_class": {k: {"triplets": v[0], "fp64": v[1], "mixed": v[2]} for k, v in sorted(per_class.items())}}
        out["reference"] = {"seconds_all_threads": t_all, "triplets_per_s_all_threads": 2000 / t_all,
                            "seconds_1_thread": t_one, "triplets_per_s_1_thread": 2000 / t_one,
                            "threads_all": nproc, "cpu_model": oracle.cpu_model(),
                            "note": "1-thread time measured on the first 200 triplets, scaled to 2000"}
    f64.close()
    mix.close()
    torch.cuda.empty_cache()
    return out


def run_mixed_vs_reference(bt, mols, pds, ads, threshold, max_dense=4e7, n_take=4):
    """The mixed-precision served/batched path against the reference library
    (oracle/_ref, FP64) per integral type and, for (mu nu|P), per class, on the
    first n_take molecules of the batch whose dense (mu nu|P) stays below
    max_dense doubles: max abs and max rel (|value| > 1e-6) error."""
    import importlib

    import numpy as np

    import oracle

    mi = importlib.import_module("electron-integral-playground_b200.molecular_integral")
    ref = oracle.reference()
    if ref is None:
        return None
    take = [i for i, m in enumerate(mols) if m.n_aux * m.n_ao * m.n_ao <= max_dense][:n_take]

    def err(a, b):
        d = np.abs(a - b)
        big = np.abs(b) > 1e-6
        return [float(d.max()) if d.size else 0.0, float((d[big] / np.abs(b[big])).max()) if big.any() else 0.0]

    def merge(acc, key, e):
        cur = acc.setdefault(key, [0.0, 0.0])
        acc[key] = [max(cur[0], e[0]), max(cur[1], e[1])]

    sub = [mols[i] for i in take], [pds[i] for i in take], [ads[i] for i in take]
    charges = [np.asarray(mols[i].geometry, dtype=np.float64) for i in take]
    b = bt.ThreeCenterBatch(*sub, precision="mixed", fp32_threshold=threshold, charges_list=charges)
    b.alloc_output()
    b.run()
    b.status()
    bm = bt.ThreeCenterBatch(sub[0], [bt.metric_pair_tables(a) for a in sub[2]], sub[2], precision="mixed",
                             fp32_threshold=threshold)
    bm.alloc_output()
    bm.run()
    bm.status()
    types, classes = {}, {}
    for k, i in enumerate(take):
        mol, pd, ad = mols[i], pds[i], ads[i]
        want = oracle.drive_three_center(ref, pd, ad, mol)
        got = b.dense(k)
        merge(types, "3c", err(got, want))
        # per class: the elements of aux shells of l_k and orbital shells of l_i, l_j
        ao_of = {}
        for (li, lj), p in pd.items():
            for l, st in ((li, p.i_ao_start), (lj, p.j_ao_start)):
                ao_of.setdefault(l, set()).update(int(s) + c for s in np.unique(st) for c in range(2 * l + 1))
        for lk, a in ad.items():
            rows = np.array(sorted({int(s) + c for s in np.unique(a.i_ao_start) for c in range(2 * lk + 1)}))
            for (li, lj) in pd:
                A, B = np.array(sorted(ao_of[li])), np.array(sorted(ao_of[lj]))
                sl = np.ix_(rows, A, B)
                merge(classes, f"{li}{lj}|{lk}", err(got[sl], want[sl]))
        merge(types, "V", err(b.dense_V(k), oracle.drive_nuclear_attraction(ref, pd, mol, charges[k])))
        merge(types, "PQ", err(bm.dense_metric(k), oracle.drive_two_center(ref, ad, mol)))
        merge(types, "S", err(mi.overlap(pd, mol), oracle.drive_overlap(ref, pd, mol)))
    b.close()
    bm.close()
    return {"molecules": take, "atoms": [len(mols[i].elements) for i in take], "fp32_threshold": threshold,
            "what": "max abs / max rel (|reference| > 1e-6) of the mixed-precision path vs the reference library; "
                    "V and (P|Q) run FP64 inside the mixed path, S is the FP64 drop-in",
            "by_type": {k: {"max_abs": v[0], "max_rel": v[1]} for k, v in types.items()},
            "by_class_3c": {k: {"max_abs": v[0], "max_rel": v[1]} for k, v in sorted(classes.items())}}


def run_reference_arm(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    mols, pds, ads, stats = build_workload(args.seed, args.molecules)
    vals = []
    for i in range(args.warmup + args.steps):
        s = reference_sample(mols, pds, ads, stats, args.ref_budget)
        if s is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference library not built (make -C oracle ref)"}))
            return
        if i >= args.warmup:
            vals.append(s)
    v = statistics.mean(x["value"] for x in vals)
    ms = statistics.mean(x["seconds"] for x in vals) * 1e3
    sample = (f"molecules {vals[0]['molecules']} of the batch (dense output <= 2e8 doubles each), "
              f"{vals[0]['triplets']} screened triplets per step")
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generators; no dataset)", "impl": "reference",
        "config": {"workload": WORKLOAD, "molecules": args.molecules, "seed": args.seed},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": vals[0]["cores"], "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--molecules", type=int, default=64)
    ap.add_argument("--ref-budget", type=float, default=12.0, help="seconds of reference CPU work per sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp32-threshold", type=float, default=1e-3,
                    help="mixed precision: FP32 for shell pairs with bound below this")
    ap.add_argument("--serve-requests", type=int, default=120, help="serving sample: requests (0 = skip)")
    ap.add_argument("--serve-rates", default="2,4,20",
                    help="serving sample: Poisson arrival rates, req/s (comma-separated)")
    ap.add_argument("--serve-alone", type=int, default=40, help="requests also timed alone in FP64")
    ap.add_argument("--no-e2e-df", dest="e2e_df", action="store_false",
                    help="e2e returns per-molecule checksums instead of the density-fitted J (profiling runs)")
    ap.add_argument("--no-water10", action="store_true", help="skip the 10-water per-type timings")
    ap.add_argument("--no-high-l", action="store_true", help="skip the 2000 high-l random triplets")
    ap.add_argument("--only-high-l", action="store_true",
                    help="time only the 2000 high-l random triplets (FP64 and mixed; the line's value is FP64 "
                         "triplets/s); for profiling the general kernel")
    ap.add_argument("--no-mixed-reference", action="store_true",
                    help="skip the mixed-precision error against the reference library")
    ap.add_argument("--no-water100", action="store_true",
                    help="skip the 100-water mixed-vs-FP64 per-class measurement")
    ap.add_argument("--tune", action="store_true",
                    help="run the autotuner on this workload first and rewrite its cache")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference_arm(args)

    import numpy as np
    import torch

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import importlib

    bt = importlib.import_module("electron-integral-playground_b200.batch")
    at = importlib.import_module("electron-integral-playground_b200.autotune")
    rf = importlib.import_module("electron-integral-playground_b200.roofline")
    lm = importlib.import_module("electron-integral-playground_b200._lib")
    if lm.lib().eip_init(local) != 0:
        raise RuntimeError(lm.lib().eip_last_error().decode())

    if args.only_high_l:
        c3 = run_random_high_l_triplets(torch, bt, bt.measure_fma_peak(), steps=args.steps, seed=args.seed, reference=False)
        if rank == 0:
            print(json.dumps({"metric": "random high-l shell triplets/s (FP64)", "value": c3["fp64"]["triplets_per_s"],
                              "unit": "triplets/s", "n_gpus": 1, "steps": args.steps, "warmup": 3,
                              "ms_per_step": c3["fp64"]["ms_per_step"], "higher_is_better": True,
                              "config": {"workload": c3["workload"]}, "random_triplets_high_l": c3}), flush=True)
        os._exit(0)
    mols, pds, ads, stats = build_workload(shard_seed(args.seed, rank), args.molecules)
    tot, per_class = rf.totals(stats)
    batch = bt.ThreeCenterBatch(mols, pds, ads, precision="fp64")
    free, _ = torch.cuda.mem_get_info()
    if batch.output_bytes > free - (2 << 30):
        raise RuntimeError(f"packed output {batch.output_bytes / 1e9:.1f} GB exceeds free device memory")
    batch.alloc_output()
    out_ptr = batch.L.eip_batch_output_device(batch.h)
    tuning = at.load()
    if args.tune:
        table, timings = at.tune(batch, sorted(per_class))
        # FP32 kernels: a mixed batch whose every shell pair takes the FP32 path
        all32 = bt.ThreeCenterBatch(mols, pds, ads, precision="mixed", fp32_threshold=float("inf"))
        all32.bind_output(out_ptr)
        table32, timings32 = at.tune(all32, sorted(per_class), fp32=True)
        all32.bind_output(0)
        all32.close()
        if rank == 0:
            at.save(table, timings, {"workload": WORKLOAD, "seed": args.seed, "molecules": args.molecules,
                                     "gpu": torch.cuda.get_device_name(local)}, table_fp32=table32,
                    timings_fp32=timings32)
        tuning = {"variants": table, "variants_fp32": table32}  # applied in-process by the tuner
    mixed = bt.ThreeCenterBatch(mols, pds, ads, precision="mixed", fp32_threshold=args.fp32_threshold)
    mixed.bind_output(out_ptr)  # same layout; the two paths run one after the other
    table_bytes = {"fp64": batch.table_bytes, "mixed": mixed.table_bytes}
    out_bytes = batch.output_bytes
    # End-to-end product: the density-fitted Coulomb matrix of every molecule
    # for a density given per step.  The (P|Q) Cholesky factors depend only on
    # the geometry and auxiliary basis (like the pair tables) and are made once
    # here; per step: tables and densities in, (mu nu|P), gamma, solve, J, J out.
    dfm = importlib.import_module("electron-integral-playground_b200.density_fitting")
    factors, shifts = [], []
    for m, ad in (zip(mols, ads) if args.e2e_df else []):
        M = dfm.metric_matrix(torch, m, ad)
        Lf, lam = dfm.metric_factor(torch, M)
        factors.append(Lf)
        shifts.append(lam / float(M.diagonal().max()))
        del M
    rng_d = np.random.default_rng(args.seed + 17)
    dens = []
    for m in mols:
        C = rng_d.standard_normal((m.n_ao, max(1, m.n_ao // 8)))
        dens.append((C @ C.T / m.n_ao).ravel())
    D_pin = torch.from_numpy(np.concatenate(dens)).pin_memory()
    D_dev = torch.empty_like(D_pin, device="cuda")

    def measure(b, clocks_path):
        """K graph launches timed with CUDA events on b's stream (value), then K
        end-to-end steps (H2D tables and densities, graph, density-fitted J of
        every molecule, D2H of J)."""
        stream = torch.cuda.ExternalStream(b.stream)
        for _ in range(args.warmup):
            b.run(sync=False)
        torch.cuda.synchronize()
        marks = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        with ClockSampler(clocks_path) as cs:
            if world > 1:
                torch.distributed.barrier()
            marks[0].record(stream)
            for k in range(args.steps):
                b.run(sync=False)
                marks[k + 1].record(stream)
            torch.cuda.synchronize()
        per_step = [marks[k].elapsed_time(marks[k + 1]) for k in range(args.steps)]
        total = marks[0].elapsed_time(marks[-1])
        if world > 1:
            total = reduce_over_ranks([total], torch.distributed.ReduceOp.MAX, "cuda")[0]
        b.status()
        if not args.e2e_df:
            # profiling runs: tables in, the graph, per-molecule checksums out
            h_ck = np.empty(len(mols))

            def e2e_ck():
                b.upload()
                b.run(checksum=True, sync=False)
                b._check(b.L.eip_batch_checksums(b.h, lm.dp(h_ck)), "checksums")

            for _ in range(2):
                e2e_ck()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                e2e_ck()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e = e0.elapsed_time(e1) / args.steps
            return {"ms": total / args.steps, "per_step": per_step, "e2e_ms": e2e, "e2e_wall_ms": e2e,
                    "clocks": cs.summary(local), "launches": b.launches_per_run * args.steps,
                    "df_gamma_ms": None, "df_coulomb_ms": None, "j_abs_sum": None,
                    "h2d": b.table_bytes, "d2h": 8 * len(mols)}
        bc = dfm.BatchCoulomb(torch, b, factors, inverse_factors=True)
        J_pin = torch.empty(bc.n_ao2, dtype=torch.float64).pin_memory()

        def e2e_step():
            b.upload()
            with torch.cuda.stream(stream):
                D_dev.copy_(D_pin, non_blocking=True)
            b.run(sync=False)
            bc.run(D_dev)
            with torch.cuda.stream(stream):
                J_pin.copy_(bc.J[:bc.n_ao2], non_blocking=True)
            stream.synchronize()

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1e3 / args.steps
        e2e = e0.elapsed_time(e1) / args.steps
        if world > 1:
            e2e = reduce_over_ranks([e2e], torch.distributed.ReduceOp.MAX, "cuda")[0]
        # the consumer stages alone (gamma, the solves, J) on the resident
        # output, CUDA events; and the solves by triangular substitution
        # (cholesky_solve) on the same gamma, for their time and difference
        g0, g1, g2, g3, g4 = (torch.cuda.Event(enable_timing=True) for _ in range(5))
        g0.record(stream)
        bc.fit(D_dev)
        g1.record(stream)
        bc.solve()
        g2.record(stream)
        bc.coulomb()
        g3.record(stream)
        tri = dfm.BatchCoulomb(torch, b, factors, inverse_factors=False)
        with torch.cuda.stream(stream):
            tri.gamma.copy_(bc.gamma)
        torch.cuda.synchronize()
        t0_ev = torch.cuda.Event(enable_timing=True)
        t0_ev.record(stream)
        tri.solve()
        g4.record(stream)
        tri.coulomb()
        torch.cuda.synchronize()
        c_scale = float(tri.c.abs().max())
        j_scale = float(tri.J.abs().max())
        solve_cmp = {"inverse_factor_ms": g1.elapsed_time(g2), "cholesky_solve_ms": t0_ev.elapsed_time(g4),
                     "max_abs_c_diff_rel": float((bc.c - tri.c).abs().max()) / max(c_scale, 1e-300),
                     "max_abs_J_diff_rel": float((bc.J - tri.J).abs().max()) / max(j_scale, 1e-300)}
        del tri
        j_check = float(J_pin.abs().sum())
        return {"ms": total / args.steps, "per_step": per_step, "e2e_ms": e2e, "e2e_wall_ms": wall,
                "clocks": cs.summary(local), "launches": b.launches_per_run * args.steps,
                "df_gamma_ms": g0.elapsed_time(g1), "df_coulomb_ms": g2.elapsed_time(g3), "j_abs_sum": j_check,
                "df_solve": solve_cmp,
                "h2d": b.table_bytes + 8 * D_pin.numel(), "d2h": 8 * bc.n_ao2}

    import tempfile

    cdir = os.environ.get("EIP_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
    cpath = lambda tag: os.path.join(cdir, f"eip_clocks_{tag}_rank{rank}_{os.getpid()}.csv")
    m64 = measure(batch, cpath("fp64"))
    mmix = measure(mixed, cpath("mixed"))
    factors.clear()  # the (P|Q) factors (about 14 GB) are not needed below
    del D_dev
    torch.cuda.empty_cache()
    split64 = split32 = 0
    for (li, lj, lk) in per_class:
        sp = mixed.precision_split(li, lj, lk)
        if sp:
            split64 += sp[0]
            split32 += sp[1]
    mixed.bind_output(0)
    mixed.close()

    # Per-class device time (each FP64 class kernel alone, 2 launches, CUDA events).
    stream = torch.cuda.ExternalStream(batch.stream)
    class_ms = {}
    for (li, lj, lk) in sorted(per_class):
        if not batch.run_class(li, lj, lk):
            continue
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(2):
            batch.run_class(li, lj, lk)
        ev1.record(stream)
        torch.cuda.synchronize()
        class_ms[(li, lj, lk)] = ev0.elapsed_time(ev1) / 2
    batch.status()
    # The dominant class's FP32 kernel (the mixed path's FP32 half) alone: a
    # batch whose every shell pair takes FP32, bound to the same output.
    dom = max(class_ms, key=class_ms.get) if class_ms else None
    fp32_dom_ms = None
    if dom:
        all32 = bt.ThreeCenterBatch(mols, pds, ads, precision="mixed", fp32_threshold=float("inf"))
        all32.bind_output(out_ptr)
        s32 = torch.cuda.ExternalStream(all32.stream)
        if all32.run_class(*dom):
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(s32)
            for _ in range(2):
                all32.run_class(*dom)
            ev1.record(s32)
            torch.cuda.synchronize()
            fp32_dom_ms = ev0.elapsed_time(ev1) / 2
        all32.status()
        all32.bind_output(0)
        all32.close()
    fp64_peak = bt.measure_fma_peak(True)
    fp32_peak = bt.measure_fma_peak(False)
    batch.close()
    torch.cuda.empty_cache()
    err = mixed_error(bt, mols, pds, ads, args.fp32_threshold, torch)
    if world > 1:  # every rank's mixed result must pass for the mixed headline
        err["max_abs"] = reduce_over_ranks([err["max_abs"]], torch.distributed.ReduceOp.MAX, "cuda")[0]
    mixed_ok = err["max_abs"] <= 1e-10
    head = mmix if mixed_ok else m64

    # whole-job units: the shards differ, so sum them over the ranks
    screened, primitive, contracted, atoms, out_elems_total = reduce_over_ranks(
        [tot["screened"], tot["primitive"], tot["contracted"], sum(len(m.elements) for m in mols), out_bytes / 8],
        torch.distributed.ReduceOp.SUM if world > 1 else None, "cuda")
    value = screened / (head["ms"] * 1e-3)
    # measured copy bandwidth of the B200s (MEASURED_PEAKS.json); without that
    # file, an earlier copy-bandwidth measurement of 6.65 TB/s ("of fallback")
    hbm_peak, hbm_source = 6650.0, "fallback 6.65 TB/s (earlier copy-bandwidth measurement on B200)"
    try:
        hbm_peak = float(json.loads((REPO / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
        hbm_source = "MEASURED_PEAKS.json hbm_gbs (measured copy bandwidth of this GPU model)"
    except Exception:
        pass
    roof = None
    if dom:
        achieved = per_class[dom]["flops"] / (class_ms[dom] * 1e-3) / 1e12
        traffic = None
        # DRAM bytes of one launch from an ncu capture on a small case of the
        # same kernel, scaled to this workload by the ratio of algorithmic bytes
        # (profiles/k3c_fast_124_traffic_small_case.md says how)
        tfile = REPO / "profiles" / "k3c_fast_124_traffic_small_case.md"
        if tfile.exists():
            for line in tfile.read_text().splitlines():
                if line.startswith(f"dram_bytes_per_launch_scaled {dom[0]}{dom[1]}{dom[2]} "):
                    traffic = float(line.split()[2])
        roof = {"bound": "fp64", "kernel": f"k3c_fast<{dom[0]},{dom[1]},{dom[2]}> (FP64)", "achieved": achieved,
                "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak, "traffic": traffic,
                "peak_source": "FP64 FMA microbenchmark on this GPU (eip_measure_fma_peak), this run",
                "algorithmic_flops_per_launch": per_class[dom]["flops"], "ms_per_launch": class_ms[dom],
                "whole_step_tflops_fp64": tot["flops"] / (m64["ms"] * 1e-3) / 1e12,
                "whole_step_frac_fp64": tot["flops"] / (m64["ms"] * 1e-3) / 1e12 / fp64_peak,
                "output_store_gbs": tot["out_bytes"] / (head["ms"] * 1e-3) / 1e9,
                "hbm_peak_gbs": hbm_peak, "output_store_frac_of_hbm": (
                    None if hbm_peak is None else tot["out_bytes"] / (head["ms"] * 1e-3) / 1e9 / hbm_peak),
                "hbm_peak_source": hbm_source,
                "fp32_kernel": None if fp32_dom_ms is None else {
                    "kernel": f"k3c_fast<{dom[0]},{dom[1]},{dom[2]}> (FP32, every shell pair)",
                    "ms_per_launch": fp32_dom_ms,
                    "achieved": per_class[dom]["flops"] / (fp32_dom_ms * 1e-3) / 1e12, "peak": fp32_peak,
                    "frac": per_class[dom]["flops"] / (fp32_dom_ms * 1e-3) / 1e12 / fp32_peak,
                    "peak_source": "FP32 FMA microbenchmark on this GPU, this run"}}
    cpu = None
    dropin = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        oracle.set_reference_threads(os.cpu_count() or 1)
        smp = reference_sample(mols, pds, ads, stats, args.ref_budget)
        if smp is not None:
            cpu = {"value": smp["value"], "unit": UNIT, "cores": smp["cores"], "kind": "reference",
                   "cpu_model": oracle.cpu_model(),
                   "sample": f"molecules {smp['molecules']} of the batch (dense output <= 2e8 doubles each), "
                             f"{smp['triplets']} screened triplets, {smp['seconds']:.1f} s, all host threads",
                   "gpu_same_sample": same_sample_rate(bt, torch, mols, pds, ads, smp, args)}
            dropin = dropin_sample(mols, pds, ads, stats, smp["molecules"])
    water10 = high_l = mixed_ref = None
    if rank == 0 and world == 1:
        if not args.no_water10:
            water10 = run_water10_per_type(args.seed)
        if not args.no_high_l:
            high_l = run_random_high_l_triplets(torch, bt, fp64_peak, seed=args.seed)
        if not args.no_mixed_reference:
            mixed_ref = run_mixed_vs_reference(bt, mols, pds, ads, args.fp32_threshold)
    serving = run_serving(args, torch, args.seed) if args.serve_requests > 0 and rank == 0 else None
    water100 = run_water100_windows(torch, bt, args.fp32_threshold, args.seed) if not args.no_water100 and rank == 0 else None
    if rank == 0:
        per = head["per_step"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32 (mixed)" if mixed_ok else "f64",
            "data": "synthetic (seeded generators; no dataset)",
            "config": {"workload": WORKLOAD, "molecules": args.molecules * world, "seed": args.seed,
                       "atoms": int(atoms),
                       "precision": "mixed" if mixed_ok else "fp64",
                       "classes": len(per_class), "primitive_triplets_per_step": int(primitive),
                       "contracted_triplets_per_step": int(contracted),
                       "screened_triplets_per_step": int(screened), "threshold": THRESHOLD,
                       "packed_output_bytes": out_bytes, "input_table_bytes": table_bytes,
                       "l2": "inputs + packed output per step exceed the 126 MB L2 (no flush needed)",
                       "parallelism": f"{world} independent shard(s)"},
            "serving_summary": None if serving is None else {
                "requests_per_rate": serving["requests"],
                "rates": [{k: r[k] for k in ("rate_rps", "throughput_rps", "latency_p50_ms", "latency_p99_ms",
                                             "latency_p99_ci_ms")}
                          for r in serving["rates"]],
                "alone_fp64_rps": serving["alone_fp64"]["throughput_rps"],
                "alone_fp64_p50_ms": serving["alone_fp64"]["latency_p50_ms"]},
            "precision": {"fp64_value": screened / (m64["ms"] * 1e-3), "fp64_ms_per_step": m64["ms"],
                          "mixed_value": screened / (mmix["ms"] * 1e-3), "mixed_ms_per_step": mmix["ms"],
                          "fp32_threshold": args.fp32_threshold,
                          "fp32_fraction_of_triplets": split32 / max(1, split32 + split64),
                          "mixed_vs_fp64_error": err, "fp32_fma_peak_tflops": fp32_peak,
                          "headline": "mixed" if mixed_ok else "fp64"},
            "integrals_per_s": {"value": out_elems_total / (head["ms"] * 1e-3),
                                "what": "spherical (mu nu|P) values written per second (packed, i<=j shell pairs)"},
            "e2e": {"value": screened / (head["e2e_ms"] * 1e-3), "unit": UNIT,
                    "h2d_bytes_per_step": head["h2d"], "d2h_bytes_per_step": head["d2h"],
                    "ms_per_step": head["e2e_ms"], "wall_ms_per_step": head["e2e_wall_ms"],
                    "fp64_value": screened / (m64["e2e_ms"] * 1e-3),
                    "result": "density-fitted Coulomb matrix J of every molecule (gamma = (mu nu|P) D, "
                              "c = (P|Q)^-1 gamma, J = (mu nu|P) c) copied to pinned host memory each step; "
                              "inputs per step: every pair/auxiliary table and the 64 densities, from pinned "
                              "host memory; (P|Q) Cholesky factors and their inverses made once per geometry "
                              "before timing (c = L^-T (L^-1 gamma))"
                              " "
                              f"({sum(1 for x in shifts if x > 0)} of {len(shifts)} metrics needed a diagonal "
                              f"shift, largest {max(shifts, default=0):.0e} x max diag)"
                              if args.e2e_df else "per-molecule checksums (--no-e2e-df profiling run)",
                    "df_kernels_ms": None if head["df_gamma_ms"] is None else {
                        "gamma": head["df_gamma_ms"], "coulomb": head["df_coulomb_ms"], "bytes_read_each": out_bytes,
                        "gamma_gbs": out_bytes / (head["df_gamma_ms"] * 1e-3) / 1e9,
                        "coulomb_gbs": out_bytes / (head["df_coulomb_ms"] * 1e-3) / 1e9,
                        "solve": head.get("df_solve")}},
            "roofline": roof, "cpu_baseline": cpu, "dropin_fp64": dropin, "serving": serving,
            "water100_mixed_vs_fp64": water100, "water10_per_type": water10, "random_triplets_high_l": high_l,
            "mixed_vs_reference": mixed_ref,
            "gpu_launches": head["launches"], "clocks": head["clocks"], "clocks_fp64": m64["clocks"],
            "latency_ms": {"p50": statistics.median(per), "p99": sorted(per)[min(len(per) - 1, int(0.99 * len(per)))],
                           "what": "per-step (whole batch) device time; request latency is under serving"},
            "class_ms": {f"{k[0]}{k[1]}|{k[2]}": round(v, 4) for k, v in sorted(class_ms.items())},
            "tuning": "autotuned variants (tuning/b200_fp64.json)" if tuning else "default variants",
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    # End the process here: the serving loop's worker threads and torch's
    # cached pinned blocks would otherwise be torn down after the CUDA context
    # at interpreter exit (an abort in a tensor destructor), failing a run
    # whose results are already printed.
    torch.cuda.synchronize()
    sys.stdout.flush()
    sys.stderr.flush()
    os._exit(0)


if __name__ == "__main__":
    main()
