"""Continuous-batching request loop for many solves of uneven size on one GPU.

A stream of requests (object, wavelength, a few incidences each) arrives over
time.  `SLOTS` worker threads each own an ifdda Context (one CUDA stream) and
take the next request in arrival order as soon as they are free *and* the
request's device footprint fits in the HBM budget next to the requests in
flight; their solves then overlap on the GPU.  Each slot keeps an LRU cache of
Green spectra keyed by (lattice, spacing, wavelength), so a repeated object
size at the same wavelength skips the spectrum build.

With `ragged=True` a free slot also takes every other request that has
arrived, whose object fits the head request's box (the smallest compiled box
holding it, padded by at most `pad_ratio` in volume) and that fits the HBM
budget, up to `max_batch_rhs` right-hand sides: they are solved as one ragged
batch (ifdda_inverserig_ragged), one launch sequence per iteration for every
right-hand side of every object, each object with its own spectrum, spacing,
wavelength and polarisability.  A request's vectors are laid out on the box's
sites, so its result does not depend on the requests it shares a batch with.

Either way every request's result is computed with fixed-order reductions, so
it is the same bit for bit alone and inside the mix.

The reference solves one object at a time (cdmlib/cdmlib.f:3-60 called from
the GUI's run thread, cdm/cdmRunWidget.cpp:162); this loop is the serving
layer the batched solver is driven by.
"""
from __future__ import annotations

import collections
import math
import threading
import time
import weakref
from dataclasses import dataclass, field

import numpy as np

from . import objects
from .api import Context, IFDDA_FP64, IFDDA_MIXED


@dataclass
class Request:
    rid: int
    shape: str             # "sphere" or "cube"
    n: int                 # lattice edge
    d: float               # spacing (m)
    eps: complex
    wavelength: float      # (m)
    incidences: list       # [(kx/k0, ky/k0, pp)]
    arrival: float = 0.0   # seconds after the stream start


@dataclass
class Result:
    rid: int
    FFloc: np.ndarray
    tol1: np.ndarray
    nloop: np.ndarray
    ncompte: np.ndarray
    nstop: int
    infostr: str
    start: float
    end: float
    arrival: float
    slot: int
    green_hit: bool
    # seconds spent in this request's (or its ragged batch's) phases: host
    # object build and device inputs, Green spectra, solve, read-back
    phases: dict = field(default_factory=dict)


def _request_inputs_bytes(N: int, nrhs: int) -> int:
    """A request's device inputs and outputs (_DeviceRequest): incident,
    dipole-moment and local fields, the (nmax,3,3) polarisability, positions,
    Tabdip and the isotropic alpha."""
    return 3 * (3 * N * 16) * nrhs + 9 * N * 16 + 3 * N * 8 + N * 4 + N * 16


def pick_next(pending, now: float, policy: str, max_wait: float):
    """The request a server serves next from `pending` (sorted by arrival,
    its head arrived by `now`): fifo takes the head; sjf takes the arrived
    request with the least work (lattice sites x incidences; the earliest of
    equals), or the head once it has waited max_wait seconds."""
    head = pending[0]
    if policy == "fifo" or now - head.arrival >= max_wait:
        return head
    best, cost = head, head.n ** 3 * len(head.incidences)
    for q in pending:
        if q.arrival > now:
            break
        c = q.n ** 3 * len(q.incidences)
        if c < cost:
            best, cost = q, c
    return best


def footprint_bytes(n: int, nrhs: int, precision: int) -> int:
    """Device bytes one solve holds: the spectrum (FP64 + FP32), mat-vec
    scratch, Krylov vectors and the request's inputs and outputs."""
    N = n ** 3
    Np = (n + 1) ** 3
    green = 6 * Np * (16 + 8)
    scr64 = 18 * N * 16 * nrhs
    vec64 = 14 * 3 * N * 16 * nrhs
    io = _request_inputs_bytes(N, nrhs) + N * 16
    # solver bookkeeping (reductions, states, captured loops) and allocator
    # granularity: 8 MiB
    extra = 8 << 20
    if precision == IFDDA_MIXED:
        return green + scr64 + 18 * N * 8 * nrhs + 14 * 3 * N * 8 * nrhs + 2 * 3 * N * 16 * nrhs + io + extra
    return green + scr64 + vec64 + io + extra


def ragged_footprint_bytes(box: int, nrhs: int, precision: int) -> int:
    """Device bytes of nrhs right-hand sides in a ragged batch on a box of
    side `box` (vectors on the box's sites), spectra not included."""
    N = box ** 3
    scr64 = 18 * N * 16 * nrhs
    vec64 = 14 * 3 * N * 16 * nrhs
    # the batch's own field copies on the box, and the request's inputs
    io = 3 * 3 * N * 16 * nrhs + 2 * N * 16 + _request_inputs_bytes(N, nrhs)
    if precision == IFDDA_MIXED:
        return scr64 + 18 * N * 8 * nrhs + 14 * 3 * N * 8 * nrhs + 2 * 3 * N * 16 * nrhs + io
    return scr64 + vec64 + io


def green_bytes(box: int) -> int:
    return 6 * (box + 1) ** 3 * (16 + 8)


COMPILED_SIDES = (1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 80, 96, 128, 160, 192, 256, 320)


def box_side(n: int) -> int:
    """Smallest side >= n whose 2n is a compiled FFT length."""
    for m in COMPILED_SIDES:
        if m >= n:
            return m
    raise ValueError(f"lattice side {n} above 320")


def make_stream(nreq: int, rate: float, seed: int = 4, edges=(16, 24, 32, 48, 64, 80, 96), max_inc: int = 32,
                d: float = 10e-9):
    """Seeded synthetic request stream: Poisson arrivals at `rate` per second,
    sphere or cube, edge uniform in `edges`, eps' ~ U[1.5, 4], eps'' ~
    U[0, 0.5], wavelength ~ U[400, 800] nm, 1..max_inc incidences uniform on
    the NA 0.9 disk, s and p alternating."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for rid in range(nreq):
        t += rng.exponential(1.0 / rate)
        ninc = int(rng.integers(1, max_inc + 1))
        rr = 0.9 * np.sqrt(rng.uniform(0, 1, ninc))
        th = rng.uniform(0, 2 * np.pi, ninc)
        inc = [(float(a * math.cos(b)), float(a * math.sin(b)), float(q % 2)) for q, (a, b) in enumerate(zip(rr, th))]
        out.append(Request(rid=rid, shape="sphere" if rng.uniform() < 0.5 else "cube",
                           n=int(edges[int(rng.integers(0, len(edges)))]), d=d,
                           eps=complex(rng.uniform(1.5, 4.0), rng.uniform(0.0, 0.5)),
                           wavelength=float(rng.uniform(400e-9, 800e-9)), incidences=inc, arrival=t))
    return out


def build_object(req: Request):
    k0 = 2 * math.pi / req.wavelength
    if req.shape == "sphere":
        ob = objects.sphere(req.n * req.d / 2, req.eps, req.n, k0, "RR", na=-1)
    else:
        ob = objects.cube(req.n * req.d, req.eps, req.n, k0, "RR")
    return ob, k0


class _PinnedPool:
    """Page-locked host buffers for the local fields read back, shared by
    every slot and server of the process.  A read-back takes the smallest
    free buffer that holds it (allocating one, rounded up to 64 MiB, only
    when none does) and the returned array gives it back when it is freed.
    Allocating page-locked memory is slow and holds the CUDA driver while it
    runs, stalling the other slots' calls; a steady request stream reuses the
    buffers instead, and prewarm() makes them before a timed stream starts."""

    GRAIN = 64 << 20

    def __init__(self, pin: bool = True):
        self.lock = threading.Lock()
        self.free = []
        self.pin = pin

    def acquire(self, nbytes: int):
        import torch
        with self.lock:
            fit = [i for i, b in enumerate(self.free) if b.numel() >= nbytes]
            if fit:
                return self.free.pop(min(fit, key=lambda i: self.free[i].numel()))
        size = -(-nbytes // self.GRAIN) * self.GRAIN
        return torch.empty(size, dtype=torch.uint8, pin_memory=self.pin)

    def release(self, buf):
        with self.lock:
            self.free.append(buf)

    def array_view(self, shape):
        """(tensor, array): a complex128 tensor of `shape` on a pool buffer
        and the numpy array on the same memory.  The buffer returns to the
        pool when the array (with every view of it) is freed, so the tensor
        must not outlive the array."""
        import torch
        nbytes = int(np.prod(shape)) * 16
        buf = self.acquire(nbytes)
        out = buf[:nbytes].view(torch.complex128).view(tuple(shape))
        arr = out.numpy()
        weakref.finalize(arr, self.release, buf)
        return out, arr

    def prewarm(self, nbytes: int, count: int):
        bufs = [self.acquire(nbytes) for _ in range(count)]
        for b in bufs:
            self.release(b)

    def clear(self):
        with self.lock:
            self.free = []


_PINNED = _PinnedPool()


def prewarm_readback(nbytes: int, count: int):
    """Make `count` page-locked read-back buffers of at least nbytes each
    (a request's local field takes 3 x dipoles x incidences x 16 bytes)."""
    _PINNED.prewarm(int(nbytes), int(count))


def release_readback_buffers():
    """Drop the free page-locked read-back buffers (those still held by
    result arrays return to the pool when the arrays are freed)."""
    _PINNED.clear()


class _Slot:
    def __init__(self, idx: int, device: int, cache_size: int):
        import torch
        self.idx = idx
        self.ctx = Context(device)
        self.dev = torch.device("cuda", device)
        # the slot's device inputs are made and read back on its context's
        # stream, so a slot waits for its own work only (no device-wide sync
        # that would wait on, or interfere with, the other slots' solves)
        self.tstream = torch.cuda.ExternalStream(self.ctx.stream(), device=self.dev)
        self.cache = collections.OrderedDict()
        self.cache_size = cache_size

    def green(self, ob, k0, box=None):
        key = (ob.nx, ob.ny, ob.nz, ob.aretecube, k0, box)
        if key in self.cache:
            self.cache.move_to_end(key)
            return self.cache[key], True
        if box is None:
            g = self.ctx.green(ob.nx, ob.ny, ob.nz, ob.aretecube, k0)
        else:
            g = self.ctx.green_box(ob.nx, ob.ny, ob.nz, (box, box, box), ob.aretecube, k0)
        self.cache[key] = g
        while len(self.cache) > self.cache_size:
            _, old = self.cache.popitem(last=False)
            old.close()
        return g, False

    def close(self):
        import torch
        # every torch block that was used on the context's stream is released
        # before the stream goes away: a cached block or pinned buffer freed
        # later would otherwise be tied to a destroyed stream
        self.tstream.synchronize()
        for g in self.cache.values():
            g.close()
        self.cache.clear()
        torch.cuda.synchronize(self.dev)
        torch.cuda.empty_cache()
        self.ctx.close()


class _DeviceRequest:
    """One request's inputs on the device (torch tensors on the slot's
    device): positions, incident fields built there, the (nmax,3,3)
    polarisability with its diagonal set from the isotropic alpha, Tabdip,
    and room for the fields.  Only the alpha, positions and Tabdip cross
    from the host; the local field is the one result read back."""

    def __init__(self, slot, req: Request):
        import torch
        ob, k0 = build_object(req)
        self.ob, self.k0 = ob, k0
        self.slot = slot
        E0, _ = objects.irradiance(1.0, 10 * req.wavelength)
        dev = slot.dev
        nb, nmax = ob.nbsphere, ob.nmax
        self.nrhs = len(req.incidences)
        with torch.cuda.stream(slot.tstream):
            self.xs = torch.from_numpy(np.ascontiguousarray(ob.xs, np.float64)).to(dev)
            self.ys = torch.from_numpy(np.ascontiguousarray(ob.ys, np.float64)).to(dev)
            self.zs = torch.from_numpy(np.ascontiguousarray(ob.zs, np.float64)).to(dev)
            alpha = torch.from_numpy(np.ascontiguousarray(ob.alpha, np.complex128)).to(dev)
            self.pol = torch.zeros(9 * nmax, dtype=torch.complex128, device=dev)
            for q in (0, 4, 8):  # (n,a,a) at n + nmax*(a + 3a)
                self.pol[q * nmax:q * nmax + nb] = alpha
            self.tab = (torch.from_numpy(np.ascontiguousarray(ob.tabdip, np.int32)).to(dev) if ob.inside_only
                        else None)
            self.ff0 = torch.empty((self.nrhs, 3 * nb), dtype=torch.complex128, device=dev)
            self.ff = torch.empty_like(self.ff0)
            self.loc = torch.empty_like(self.ff0)
        slot.tstream.synchronize()
        kx = [a * k0 for a, _, _ in req.incidences]
        ky = [b * k0 for _, b, _ in req.incidences]
        pp = [c for _, _, c in req.incidences]
        slot.ctx.planewaves_device(nb, self.xs.data_ptr(), self.ys.data_ptr(), self.zs.data_ptr(), k0, E0,
                                   [1] * len(kx), kx, ky, pp, self.ff0.data_ptr())

    @property
    def tab_ptr(self):
        return self.tab.data_ptr() if self.tab is not None else None

    def local_field(self) -> np.ndarray:
        """The local field read back to the host, on the slot's stream, into
        a page-locked buffer of the read-back pool that the returned array
        holds: the copy runs at PCIe speed and needs no second copy on the
        host (a pageable destination would cost a host-side pass and
        first-touch page faults over the whole field).  When the array is
        freed the buffer returns to the pool."""
        import torch
        out, arr = _PINNED.array_view(self.loc.shape)
        # a blocking copy: no event of the slot's stream is tied to the
        # buffer (the stream is destroyed with the slot)
        with torch.cuda.stream(self.slot.tstream):
            out.copy_(self.loc, non_blocking=False)
        return arr


def solve_request(slot: _Slot, req: Request, precision: int, tol: float = 1e-4, methodeit: str = "GPBICG1"):
    """One request on its own: incident fields built on the device, the
    batched solve of its incidences on device buffers, the local field read
    back.  Returns (result dict, green_hit)."""
    t0 = time.perf_counter()
    d = _DeviceRequest(slot, req)
    ob = d.ob
    t1 = time.perf_counter()
    g, hit = slot.green(ob, d.k0)
    t2 = time.perf_counter()
    r = g.inverserig_device(d.nrhs, ob.nbsphere, ob.nmax, d.tab_ptr, d.pol.data_ptr(), d.ff0.data_ptr(),
                            d.ff.data_ptr(), d.loc.data_ptr(), methodeit, tol, precision=precision)
    t3 = time.perf_counter()
    FFloc = d.local_field()
    t4 = time.perf_counter()
    # a cached spectrum keeps no workspace: the HBM budget covers in-flight solves only
    g.release_workspace()
    t5 = time.perf_counter()
    return dict(FFloc=FFloc, tol1=r["tol1"], nloop=r["nloop"], ncompte=r["ncompte"], nstop=r["nstop"],
                infostr=r["infostr"], phases=dict(inputs=t1 - t0, green=t2 - t1, solve=t3 - t2,
                                                  readback=t4 - t3, release=t5 - t4)), hit


def solve_ragged(slot: _Slot, reqs, box: int, precision: int, tol: float = 1e-4, methodeit: str = "GPBICG1"):
    """One ragged batch on the device: every request's object on the common
    box side `box`.  Returns one (result dict, green_hit) per request."""
    items, hits, dreqs = [], [], []
    t_in = t_gr = 0.0
    for req in reqs:
        t0 = time.perf_counter()
        d = _DeviceRequest(slot, req)
        t1 = time.perf_counter()
        g, hit = slot.green(d.ob, d.k0, box)
        t_in += t1 - t0
        t_gr += time.perf_counter() - t1
        items.append((g, d.ob.nbsphere, d.ob.nmax, d.tab_ptr, d.pol.data_ptr(), d.ff0.data_ptr(), d.ff.data_ptr(),
                      d.loc.data_ptr(), d.nrhs))
        hits.append(hit)
        dreqs.append(d)
    t2 = time.perf_counter()
    tol1, nloop, ncompte, nstop, info = slot.ctx.inverserig_ragged_device(items, methodeit, tol,
                                                                          precision=precision)
    t3 = time.perf_counter()
    out, r0 = [], 0
    locs = [d.local_field() for d in dreqs]
    t4 = time.perf_counter()
    items[0][0].release_workspace()
    ph = dict(inputs=t_in, green=t_gr, solve=t3 - t2, readback=t4 - t3, release=time.perf_counter() - t4)
    for d, hit, loc in zip(dreqs, hits, locs):
        sl = slice(r0, r0 + d.nrhs)
        ok = bool(np.all(tol1[sl] < tol))
        out.append((dict(FFloc=loc, tol1=tol1[sl].copy(), nloop=nloop[sl].copy(), ncompte=ncompte[sl].copy(),
                         nstop=0 if (nstop == 0 or ok) else nstop, infostr=info, phases=ph), hit))
        r0 += d.nrhs
    return out


class Server:
    """Admission by HBM footprint + `slots` concurrent workers; with `ragged`
    each worker solves every compatible arrived request in one ragged batch."""

    def __init__(self, slots: int = 4, device: int = 0, hbm_budget: float = 120e9, precision: int = IFDDA_MIXED,
                 cache_size: int = 4, ragged: bool = False, max_batch_rhs: int = 64, max_objects: int = 64,
                 pad_ratio: float = 1.0, policy: str = "fifo", max_wait: float = 5.0):
        if policy not in ("fifo", "sjf"):
            raise ValueError("policy must be 'fifo' or 'sjf'")
        if policy == "sjf" and ragged:
            raise ValueError("the sjf policy applies to per-request serving")
        self.slots = [_Slot(i, device, cache_size if not ragged else max(cache_size, max_objects))
                      for i in range(slots)]
        # fifo: the oldest request first.  sjf: among the arrived requests the
        # one with the least work (lattice sites x incidences) first, unless
        # the oldest has waited max_wait seconds, which then goes first (so a
        # large request is delayed by at most about max_wait)
        self.policy = policy
        self.max_wait = max_wait
        self.budget = hbm_budget
        self.precision = precision
        self.in_use = 0.0
        self.cv = threading.Condition()
        self.ragged = ragged
        self.max_batch_rhs = max_batch_rhs
        self.max_objects = max_objects
        self.pad_ratio = pad_ratio

    def close(self):
        for s in self.slots:
            s.close()

    def run(self, requests, realtime: bool = True, keep_fields: bool = True):
        """Serve `requests` (sorted by arrival); returns the Results in id
        order.  With realtime, a request becomes visible at its arrival time.
        Without keep_fields every local field is still read back to the host
        but dropped once its request completes (a long stream's fields would
        otherwise all stay in host memory)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        results = {}
        t0 = time.perf_counter()
        lock = threading.Lock()

        def next_request():
            # admission: the policy's pick waits until it has arrived and its
            # footprint fits next to the work in flight
            with self.cv:
                while True:
                    if not pending:
                        return None, 0.0
                    now = time.perf_counter() - t0
                    head = pending[0]
                    arrived = (not realtime) or head.arrival <= now
                    if arrived:
                        head = pick_next(pending, now if realtime else math.inf, self.policy, self.max_wait)
                    fp = footprint_bytes(head.n, len(head.incidences), self.precision)
                    fits = self.in_use + fp <= self.budget or self.in_use == 0
                    if arrived and fits:
                        pending.remove(head)
                        self.in_use += fp
                        return head, fp
                    wait = max(0.0005, head.arrival - now) if not arrived else 0.05
                    self.cv.wait(timeout=wait)

        def next_batch():
            # the head request as above, then every arrived request that fits
            # its box (volume padding <= pad_ratio), the budget and the caps
            with self.cv:
                while True:
                    if not pending:
                        return [], 0, 0.0
                    head = pending[0]
                    now = time.perf_counter() - t0
                    box = box_side(head.n)
                    fp = ragged_footprint_bytes(box, len(head.incidences), self.precision) + green_bytes(box)
                    arrived = (not realtime) or head.arrival <= now
                    fits = self.in_use + fp <= self.budget or self.in_use == 0
                    if arrived and fits:
                        break
                    wait = max(0.0005, head.arrival - now) if not arrived else 0.05
                    self.cv.wait(timeout=wait)
                batch = [pending.popleft()]
                nr = len(head.incidences)
                keep = collections.deque()
                while pending and len(batch) < self.max_objects:
                    q = pending.popleft()
                    if realtime and q.arrival > now:
                        keep.append(q)
                        break
                    qfp = ragged_footprint_bytes(box, len(q.incidences), self.precision) + green_bytes(box)
                    ok = (box_side(q.n) == box or (q.n <= box and box ** 3 <= self.pad_ratio * q.n ** 3))
                    if ok and nr + len(q.incidences) <= self.max_batch_rhs and self.in_use + fp + qfp <= self.budget:
                        batch.append(q)
                        nr += len(q.incidences)
                        fp += qfp
                    else:
                        keep.append(q)
                while keep:
                    pending.appendleft(keep.pop())
                self.in_use += fp
                return batch, box, fp

        def worker_ragged(slot: _Slot):
            while True:
                batch, box, fp = next_batch()
                if not batch:
                    return
                start = time.perf_counter() - t0
                try:
                    outs = solve_ragged(slot, batch, box, self.precision)
                finally:
                    with self.cv:
                        self.in_use -= fp
                        self.cv.notify_all()
                end = time.perf_counter() - t0
                with lock:
                    for req, (r, hit) in zip(batch, outs):
                        results[req.rid] = Result(req.rid, r["FFloc"] if keep_fields else None, r["tol1"], r["nloop"], r["ncompte"],
                                                  r["nstop"], r["infostr"], start, end,
                                                  req.arrival if realtime else 0.0, slot.idx, hit, r["phases"])

        def worker(slot: _Slot):
            while True:
                req, fp = next_request()
                if req is None:
                    return
                start = time.perf_counter() - t0
                try:
                    r, hit = solve_request(slot, req, self.precision)
                finally:
                    with self.cv:
                        self.in_use -= fp
                        self.cv.notify_all()
                end = time.perf_counter() - t0
                with lock:
                    results[req.rid] = Result(req.rid, r["FFloc"] if keep_fields else None, r["tol1"], r["nloop"],
                                              r["ncompte"], r["nstop"],
                                              r["infostr"], start, end, req.arrival if realtime else 0.0, slot.idx,
                                              hit, r["phases"])

        target = worker_ragged if self.ragged else worker
        errors = []

        def guarded(slot: _Slot):
            # a failing worker stops the stream: the other workers finish
            # their request in flight, take no new one, and run() raises
            try:
                target(slot)
            except BaseException as e:  # noqa: B902 - re-raised by run()
                with self.cv:
                    errors.append(e)
                    pending.clear()
                    self.cv.notify_all()

        threads = [threading.Thread(target=guarded, args=(s,), daemon=True) for s in self.slots]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        if errors:
            raise errors[0]
        return [results[k] for k in sorted(results)]


def latency_stats(results, wall: float):
    lat = np.array([r.end - r.arrival for r in results])
    nrhs = sum(len(np.atleast_1d(r.tol1)) for r in results)
    # phase seconds summed over solves (a ragged batch counted once)
    batches = {}
    for r in results:
        batches[(r.slot, r.start)] = r.phases
    phase_s = {}
    for ph in batches.values():
        for k, v in ph.items():
            phase_s[k] = phase_s.get(k, 0.0) + v
    return dict(p50_ms=float(np.percentile(lat, 50) * 1e3), p99_ms=float(np.percentile(lat, 99) * 1e3),
                requests_per_s=len(results) / wall, solves_per_s=nrhs / wall,
                failed=int(sum(r.nstop != 0 for r in results)), batches=len(batches),
                phase_seconds={k: round(v, 3) for k, v in phase_s.items()})
