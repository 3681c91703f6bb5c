"""Continuous-batching integral server (device-resident request loop).

A request is one molecule asking for S, V, (P|Q) and (mu nu|P); it may carry
its pair and auxiliary tables (the C-ABI formats) or leave them to the server,
which builds them after arrival (pair tables on the device, on builder
threads).  The server

* splits each request into device pieces: (mu nu|P) with V (one slot: the
  pair tables against the auxiliary basis and against the nuclei as
  point-charge ket) and (P|Q) (the one-centre metric as pair classes
  (0, l_P), `batch.metric_pair_tables`).  A (mu nu|P) too large for one piece
  (a 200-atom molecule's packed (mu nu|P) alone is ~580 GB) becomes windows of
  auxiliary shells over ONE resident batch of the request (V in its first
  window): its tables are built and uploaded once and stay on the device until
  its last window retires;
* admits pieces in arrival order whenever the device arena (one allocation of
  `budget_bytes`, first-fit sub-allocated) has room for their packed output,
  so requests that arrive while others run are admitted as memory frees up;
* batches the whole pieces admitted at one moment into ONE batch (one
  CUDA-graph launch over all their classes) on its own stream, and launches a
  window alone on its request's resident batch; up to `max_inflight` launches
  are queued on the device (with `serialize`, the default, each waits on the
  device for the previous one, so the GPU runs one batch at a time while the
  next ones are built and queued);
* when a launch completes, hands each of its pieces' packed class blocks
  (device views into the arena) to `consumer(request, piece, blocks)` on a
  consumer stream (default: a per-request digest, sum of squares, on the
  device), and frees the launch's arena range once the consumer's work has
  finished — the loop never waits for it; S comes from the drop-in overlap
  entry point on a worker thread while the GPU works.

Latency of a request = the later of its last piece's consumption and its S,
minus its arrival.
Precision "mixed" uses the batch's FP32 gate for (mu nu|P) (<= 1e-10 of FP64,
tested); V and (P|Q) are always FP64.
"""

import collections
import concurrent.futures
import queue
import threading
import time

import numpy as np

from .batch import POINT_CHARGES, ThreeCenterBatch, metric_pair_tables


def aux_slices(aux_data, n_aux, max_functions):
    """Split the auxiliary tables into slices of whole shells, at most
    max_functions functions each (one shell at least), starts rebased to the
    slice.  Returns [(first function, end function, tables)]."""
    from .data_structure import PrimitivePairData

    starts = np.unique(np.concatenate([np.asarray(a.i_ao_start) for a in aux_data.values()]))
    edges = [0]
    for s in starts:
        if s - edges[-1] >= max_functions:
            edges.append(int(s))
    edges.append(n_aux)
    slices = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        sub = {}
        for l, a in aux_data.items():
            st = np.asarray(a.i_ao_start)
            sel = (st >= lo) & (st < hi)
            if sel.any():
                sub[l] = PrimitivePairData(P_p=None, A_a=np.ascontiguousarray(np.asarray(a.A_a)[sel]), B_b=None,
                                           coefficient=np.ascontiguousarray(np.asarray(a.coefficient)[sel]),
                                           i_ao_start=(st[sel] - lo).astype(np.int32), j_ao_start=None,
                                           i_atom=None, j_atom=None)
        if sub:
            slices.append((lo, hi, sub))
    return slices


def _n_shell_pairs(p):
    key = np.asarray(p.i_ao_start).astype(np.int64) * (1 << 32) + np.asarray(p.j_ao_start)
    return len(np.unique(key))


def packed_elems(pair_data, aux_data, n_charge=0, n_sp=None):
    """Doubles of the packed spherical output of one molecule slot (n_sp: the
    shell-pair count per pair class, if already known)."""
    total = 0
    n_aux_sh = {l: len(np.unique(np.asarray(a.i_ao_start))) for l, a in aux_data.items()}
    for (li, lj), p in pair_data.items():
        nsp = n_sp[(li, lj)] if n_sp is not None else _n_shell_pairs(p)
        for lk, nax in n_aux_sh.items():
            total += nsp * (2 * li + 1) * (2 * lj + 1) * (2 * lk + 1) * nax
        total += nsp * (2 * li + 1) * (2 * lj + 1) * n_charge
    return total


def window_edges(aux_data, n_aux, max_functions):
    """Auxiliary-function edges of windows of whole shells, at most
    max_functions functions each (one shell at least)."""
    starts = np.unique(np.concatenate([np.asarray(a.i_ao_start) for a in aux_data.values()]))
    edges = [0]
    for s in starts:
        if s - edges[-1] >= max_functions:
            edges.append(int(s))
    edges.append(n_aux)
    return edges


def window_elems(pair_sp, aux_starts, lo, hi):
    """Doubles of the packed output of the auxiliary window [lo, hi).
    pair_sp: {(l_i, l_j): shell pairs}; aux_starts: {l_k: sorted shell starts}."""
    total = 0
    for lk, st in aux_starts.items():
        nax = int(np.searchsorted(st, hi) - np.searchsorted(st, lo))
        for (li, lj), nsp in pair_sp.items():
            total += nsp * (2 * li + 1) * (2 * lj + 1) * (2 * lk + 1) * nax
    return total


class Request:
    """One molecule's integrals.  pair_data / aux_data: the C-ABI tables, or
    None to have the server build them (pair tables on the device) when the
    request arrives."""

    def __init__(self, rid, molecule, pair_data=None, aux_data=None, arrival=0.0):
        self.rid = rid
        self.molecule = molecule
        self.pair_data = pair_data
        self.aux_data = aux_data
        self.arrival = arrival
        self.pieces_left = 0
        self.digest = 0.0
        self.digest_dev = None  # device accumulator of the default consumer
        self.done = None
        self.S = None
        self.resident = None  # the resident batch of a windowed request (or its pending build)
        self.windows_left = 0
        self.charges = None
        self.tables = None  # pending table build

class Piece:
    """One molecule slot of a batch: kind "3c" ((mu nu|P) of the auxiliary
    shells from function aux_lo, with V when it carries the charges; a window
    of the request's resident batch when window is set) or "metric" (columns
    of (P|Q) from function aux_lo)."""

    def __init__(self, request, kind, pair_data, aux_data, aux_lo, elems, charges=None, aux_hi=None,
                 window=False):
        self.request = request
        self.kind = kind
        self.pair_data = pair_data
        self.aux_data = aux_data
        self.aux_lo = aux_lo
        self.aux_hi = aux_hi
        self.window = window  # computed as a window of the request's resident batch
        self.elems = elems
        self.charges = charges

    def classes(self):
        for (li, lj) in self.pair_data:
            for lk in self.aux_data:
                yield li, lj, lk
            if self.charges is not None:
                yield li, lj, POINT_CHARGES


class Arena:
    """First-fit sub-allocator over one device buffer (offsets in doubles,
    256-byte granules)."""

    def __init__(self, torch, n_doubles):
        self.buf = torch.empty(int(n_doubles), dtype=torch.float64, device="cuda")
        self.free = [(0, int(n_doubles))]

    def alloc(self, n):
        n = (int(n) + 31) & ~31
        for i, (off, size) in enumerate(self.free):
            if size >= n:
                self.free[i] = (off + n, size - n)
                if self.free[i][1] == 0:
                    self.free.pop(i)
                return off, n
        return None

    def release(self, off, n):
        self.free.append((off, n))
        self.free.sort()
        merged = []
        for o, s in self.free:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + s)
            else:
                merged.append((o, s))
        self.free = merged

    @property
    def largest_free(self):
        return max((s for _, s in self.free), default=0)

    @property
    def capacity(self):
        return self.buf.numel()


def default_consumer(request, piece, blocks):
    """blocks: [((l_i, l_j, l_k), device view of the packed block)] of one piece;
    adds the sum of squares of every value (one read of each block) to the
    request's device-side digest, without waiting for it."""
    if blocks:
        part = sum(v.dot(v) for _, v in blocks)
        request.digest_dev = part if request.digest_dev is None else request.digest_dev + part


class IntegralServer:
    def __init__(self, budget_bytes=150e9, precision="mixed", max_inflight=3, slice_fraction=0.25,
                 consumer=default_consumer, host_overlap=True, keep_blocks=False, fp32_threshold=None,
                 serialize=True, max_resident=2, dead_bytes_max=4e9):
        import torch

        self.torch = torch
        self.arena = Arena(torch, budget_bytes / 8)
        self.precision = precision
        self.fp32_threshold = fp32_threshold
        self.max_inflight = max_inflight
        # serialize: each launch waits (on the device) for the previous one, so
        # the GPU runs one batch at a time while later batches are built and
        # queued; persistent kernels of different batches sharing the GPU slow
        # each other down
        self.serialize = serialize
        self._last_ev = None
        self.slice_elems = int(self.arena.capacity * slice_fraction)
        self.consumer = consumer
        self.host_overlap = host_overlap
        self.keep_blocks = keep_blocks
        self.kept = collections.defaultdict(dict)
        self.launches = 0
        # finished batches: destroyed while nothing is in flight, because
        # freeing device memory synchronises the whole device, or once they
        # hold more than dead_bytes_max of device memory
        self._dead = []
        self.dead_bytes_max = dead_bytes_max
        self._dead_bytes = 0
        # resident batches of windowed requests (their tables and E tables stay
        # on the device, outside the arena, until the last window retires): at
        # most max_resident exist or are being built; later windowed requests
        # wait in arrival order, so a stream of large requests cannot fill the
        # device with tables of requests whose windows are far from running
        self.max_resident = max_resident
        self._resident_wait = collections.deque()
        self._n_resident = 0
        self._dead_resident = 0
        self.resident_high = 0  # most resident batches alive or being built at once
        # launches whose consumer work is queued: (event, off, alloc, pieces)
        self._consuming = []
        # requests whose device pieces are done, waiting for S
        self._awaiting_s = []
        self.cstream = torch.cuda.Stream()
        # host seconds spent planning pieces, building batches, retiring launches
        self.host_s = {"plan": 0.0, "build": 0.0, "retire": 0.0}

    # -- request decomposition -------------------------------------------------
    def _sliced(self, req, kind, pair_data):
        mol = req.molecule
        full = packed_elems(pair_data, req.aux_data)
        if full <= self.slice_elems:
            return [Piece(req, kind, pair_data, req.aux_data, 0, full)]
        width = max(1, int(self.slice_elems / (full / mol.n_aux)))
        return [Piece(req, kind, pair_data, sub, lo, packed_elems(pair_data, sub))
                for lo, hi, sub in aux_slices(req.aux_data, mol.n_aux, width)]

    def pieces_of(self, req):
        mol = req.molecule
        pair_sp = {k: _n_shell_pairs(p) for k, p in req.pair_data.items()}
        charges = np.asarray(mol.geometry, np.float64).reshape(-1, 3)
        v_elems = packed_elems(req.pair_data, {}, len(charges), n_sp=pair_sp)
        full = packed_elems(req.pair_data, req.aux_data, n_sp=pair_sp)
        if full + v_elems <= self.slice_elems:
            out = [Piece(req, "3c", req.pair_data, req.aux_data, 0, full + v_elems, charges=charges)]
        else:
            req.charges = charges
            starts = {l: np.unique(np.asarray(a.i_ao_start)) for l, a in req.aux_data.items()}
            width = max(1, int(self.slice_elems / ((full + v_elems) / mol.n_aux)))
            edges = window_edges(req.aux_data, mol.n_aux, width)
            out = [Piece(req, "3c", req.pair_data, req.aux_data, lo,
                         window_elems(pair_sp, starts, lo, hi) + (v_elems if k == 0 else 0),
                         charges=charges if k == 0 else None, aux_hi=hi, window=True)
                   for k, (lo, hi) in enumerate(zip(edges[:-1], edges[1:]))]
            req.windows_left = len(out)
        out += self._sliced(req, "metric", metric_pair_tables(req.aux_data))
        for p in out:
            if p.elems > self.arena.capacity:
                raise ValueError(f"request {req.rid}: one auxiliary shell slice exceeds the HBM budget")
        return out

    @staticmethod
    def _build_tables(req):
        """Pair tables on the device, auxiliary tables on the host (builder thread)."""
        from .device_pairs import form_pair_data_device
        from .pair_utility import form_auxiliary_pair_data

        req.pair_data = form_pair_data_device(req.molecule, 1e-14)
        req.aux_data = form_auxiliary_pair_data(req.molecule)
        return req

    def _build_resident(self, req, device):
        """Resident batch of a windowed request (runs on the builder thread)."""
        self.torch.cuda.set_device(device)
        kw = {} if self.fp32_threshold is None else {"fp32_threshold": self.fp32_threshold}
        return ThreeCenterBatch([req.molecule], [req.pair_data], [req.aux_data], precision=self.precision,
                                charges_list=[req.charges], **kw)

    # -- S on a worker thread ----------------------------------------------------
    def _host_worker(self, q):
        from .molecular_integral import overlap

        while True:
            req = q.get()
            if req is None:
                return
            try:
                req.S = overlap(req.pair_data, req.molecule)
            except Exception as exc:  # reported by the loop, which must not wait forever
                req.S = exc

    # -- the loop ------------------------------------------------------------------
    def serve(self, requests, realtime=True):
        """Serve `requests` (each with .arrival seconds from start); returns stats.
        realtime=False admits every request at once (arrival ignored)."""
        todo = collections.deque(sorted(requests, key=lambda r: r.arrival))
        preparing = []  # arrived, tables being built
        arrived = collections.deque()  # arrived with tables, not yet split
        waiting = collections.deque()  # pieces of arrived requests, FIFO
        inflight = []
        hostq = queue.Queue()
        worker = threading.Thread(target=self._host_worker, args=(hostq,), daemon=True)
        if self.host_overlap:
            worker.start()
        # resident batches of windowed requests are built on a builder thread
        # as the requests arrive; launches (a batch build + graph launch, or a
        # window) run in admission order on a launcher thread; both overlap the
        # loop and the GPU
        device = self.torch.cuda.current_device()
        init = (lambda: self.torch.cuda.set_device(device))
        builder = concurrent.futures.ThreadPoolExecutor(max_workers=2, initializer=init)
        launcher = concurrent.futures.ThreadPoolExecutor(max_workers=1, initializer=init)
        t0 = time.perf_counter()
        finished = []
        n_total = len(todo)
        try:
            while len(finished) < n_total:
                now = time.perf_counter() - t0
                while todo and (todo[0].arrival <= now or not realtime):
                    req = todo.popleft()
                    if not realtime:
                        req.arrival = now
                    if req.pair_data is None or req.aux_data is None:
                        req.tables = builder.submit(self._build_tables, req)
                        preparing.append(req)
                    else:
                        arrived.append(req)
                for req in [r for r in preparing if r.tables.done()]:
                    preparing.remove(req)
                    req.tables.result()  # re-raises a failed build
                    arrived.append(req)
                while arrived:
                    req = arrived.popleft()
                    tp = time.perf_counter()
                    ps = self.pieces_of(req)
                    self.host_s["plan"] += time.perf_counter() - tp
                    req.pieces_left = len(ps)
                    if req.windows_left:
                        self._resident_wait.append(req)
                    waiting.extend(ps)
                    if self.host_overlap:
                        hostq.put(req)
                for fut in list(inflight):
                    if fut.done() and fut.result()[1].query():
                        tr = time.perf_counter()
                        self._retire(fut.result())
                        self.host_s["retire"] += time.perf_counter() - tr
                        inflight.remove(fut)
                for entry in list(self._consuming):
                    if entry[0].query():
                        self._consumed(entry, finished, t0)
                        self._consuming.remove(entry)
                if self._awaiting_s:
                    self._finish_ready(finished, t0)
                if self._resident_wait and self._n_resident >= self.max_resident and self._dead_resident:
                    self._close_dead()  # retired resident batches make room for the next one
                while self._resident_wait and self._n_resident < self.max_resident:
                    req = self._resident_wait.popleft()
                    req.resident = builder.submit(self._build_resident, req, device)
                    self._n_resident += 1
                    self.resident_high = max(self.resident_high, self._n_resident)
                if self._dead and ((not inflight and not self._consuming) or len(self._dead) > 64
                                   or self._dead_bytes > self.dead_bytes_max):
                    self._close_dead()
                if waiting and len(inflight) < self.max_inflight:
                    largest = self.arena.largest_free
                    group, total = [], 0
                    if waiting[0].window:
                        # a window runs on its request's resident batch, once that is being built
                        if waiting[0].request.resident is not None and waiting[0].elems + 32 <= largest:
                            group.append(waiting.popleft())
                            total = group[0].elems
                    else:
                        while (waiting and not waiting[0].window
                               and total + waiting[0].elems + 32 * (len(group) + 1) <= largest):
                            p = waiting.popleft()
                            group.append(p)
                            total += p.elems
                    if group:
                        off, alloc = self.arena.alloc(total + 32 * len(group))
                        if group[0].window:
                            inflight.append(launcher.submit(self._launch_window, group[0], off, alloc))
                        else:
                            inflight.append(launcher.submit(self._launch, group, off, alloc))
                        continue
                    if not inflight and not self._consuming:
                        raise RuntimeError("a piece does not fit the empty arena")
                if not inflight and not waiting and not preparing and todo and realtime:
                    time.sleep(max(0.0, min(0.002, todo[0].arrival - (time.perf_counter() - t0))))
                else:
                    time.sleep(0.0002)
        finally:
            launcher.shutdown(wait=True)
            items = [f.result() for f in inflight if f.exception() is None]
            for item in items:
                item[0].sync()
            for item in items:
                item[0].close()
            self.cstream.synchronize()
            self._consuming.clear()
            self._close_dead()
            builder.shutdown(wait=True)
            for r in requests:
                if r.resident is not None:
                    b = r.resident.result() if isinstance(r.resident, concurrent.futures.Future) else r.resident
                    b.close()
                    r.resident = None
            self._resident_wait.clear()
            self._n_resident = self._dead_resident = 0
            if self.host_overlap:
                hostq.put(None)
                worker.join()
        wall = time.perf_counter() - t0
        lat = np.array([r.done - r.arrival for r in finished])
        # 95% bootstrap intervals of the percentiles (seeded resampling of the
        # requests' latencies): the sampling spread of p50 / p99 at this size
        boot = np.random.default_rng(0).choice(lat, size=(1000, lat.size), replace=True)
        ci = {q: [float(x) for x in np.percentile(np.percentile(boot, q, axis=1), [2.5, 97.5])] for q in (50, 99)}
        return {"requests": n_total, "wall_s": wall, "throughput_rps": n_total / wall,
                "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
                "latency_p50_ci_s": ci[50], "latency_p99_ci_s": ci[99],
                "latency_mean_s": float(lat.mean()), "launches": self.launches,
                "host_s": {k: round(v, 3) for k, v in self.host_s.items()}}

    def _launch(self, group, off, alloc):
        """One batch (one CUDA-graph launch) over every piece of the group, its
        output bound to the group's arena range; returns the in-flight record.
        Runs on the launcher thread."""
        torch = self.torch
        tb = time.perf_counter()
        kw = {} if self.fp32_threshold is None else {"fp32_threshold": self.fp32_threshold}
        b = ThreeCenterBatch([p.request.molecule for p in group], [p.pair_data for p in group],
                             [p.aux_data for p in group], precision=self.precision,
                             charges_list=[p.charges for p in group], **kw)
        if b.output_elems != sum(p.elems for p in group):
            b.close()
            raise RuntimeError("packed output size differs from the planned size")
        b.bind_output(self.arena.buf.data_ptr() + 8 * off)
        self._after_previous(b)
        b.run(sync=False)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.ExternalStream(b.stream))
        self._last_ev = ev
        self.launches += 1
        layout = [self._layout(p, lambda li, lj, lk, m=m: b.block(m, li, lj, lk)) for m, p in enumerate(group)]
        self.host_s["build"] += time.perf_counter() - tb
        return (b, ev, group, off, alloc, layout)

    def _launch_window(self, piece, off, alloc):
        """One auxiliary window of a large request on its resident batch (built
        on the builder thread).  Runs on the launcher thread."""
        torch = self.torch
        tb = time.perf_counter()
        req = piece.request
        if isinstance(req.resident, concurrent.futures.Future):
            req.resident = req.resident.result()
        b = req.resident
        n = b.window([piece.aux_lo], [piece.aux_hi], with_charges=piece.charges is not None)
        if n != piece.elems:
            raise RuntimeError("window output size differs from the planned size")
        layout = [self._layout(piece, lambda li, lj, lk: b.window_block(0, li, lj, lk))]
        self._after_previous(b)
        b.run_window(self.arena.buf.data_ptr() + 8 * off)
        ev = torch.cuda.Event()
        ev.record(torch.cuda.ExternalStream(b.stream))
        self._last_ev = ev
        self.launches += 1
        self.host_s["build"] += time.perf_counter() - tb
        return (b, ev, [piece], off, alloc, layout)

    def _after_previous(self, b):
        """With serialize, order b's next launch after the previous launch."""
        if self.serialize and self._last_ev is not None:
            self.torch.cuda.ExternalStream(b.stream).wait_event(self._last_ev)

    @staticmethod
    def _layout(piece, block_of):
        """[(class, offset, length)] of a piece's blocks in its launch's output."""
        out = []
        for li, lj, lk in piece.classes():
            blk = block_of(li, lj, lk)
            if blk is None:
                continue
            o, nsp, nax = blk
            out.append(((li, lj, lk), o, nsp * (2 * li + 1) * (2 * lj + 1) * (2 * max(lk, 0) + 1) * nax))
        return out

    def _retire(self, item):
        """A launch has completed: queue the consumer's work on the consumer
        stream (the completion event has been seen, so the output is final; no
        stream wait, since a windowed batch's stream may already hold its next
        window) and remember when that work will have finished."""
        batch, _, pieces, off, alloc, layout = item
        torch = self.torch
        with torch.cuda.stream(self.cstream):
            for p, lay in zip(pieces, layout):
                blocks = [(c, self.arena.buf[off + o:off + o + n]) for c, o, n in lay]
                self.consumer(p.request, p, blocks)
                if self.keep_blocks:
                    for c, v in blocks:
                        self.kept[p.request.rid][(p.kind, p.aux_lo) + c] = v.cpu().numpy().copy()
            ev = torch.cuda.Event()
            ev.record(self.cstream)
        self._consuming.append((ev, off, alloc, pieces))
        if pieces[0].window:
            req = pieces[0].request
            req.windows_left -= 1
            if req.windows_left == 0:  # its last window: free the tables later
                self._dead.append(batch)
                self._dead_bytes += batch.device_bytes
                self._dead_resident += 1
                req.resident = None
        else:
            batch.bind_output(0)
            self._dead.append(batch)
            self._dead_bytes += batch.device_bytes

    def _consumed(self, entry, finished, t0):
        """The consumer's work on a launch's output has finished: free the arena
        range; a request is done when its last piece is and its S (worker
        thread) is ready."""
        _, off, alloc, pieces = entry
        self.arena.release(off, alloc)
        for p in pieces:
            p.request.pieces_left -= 1
            if p.request.pieces_left == 0:
                if p.request.digest_dev is not None:
                    p.request.digest = float(p.request.digest_dev)
                self._awaiting_s.append(p.request)
        self._finish_ready(finished, t0)

    def _finish_ready(self, finished, t0):
        for req in [r for r in self._awaiting_s if r.S is not None or not self.host_overlap]:
            if isinstance(req.S, Exception):
                raise RuntimeError(f"request {req.rid}: overlap failed") from req.S
            self._awaiting_s.remove(req)
            req.done = time.perf_counter() - t0
            finished.append(req)

    def _close_dead(self):
        """Check the self-check words of finished batches and destroy them."""
        for b in self._dead:
            b.status()
            b.close()
        self._dead.clear()
        self._dead_bytes = 0
        self._n_resident -= self._dead_resident
        self._dead_resident = 0
