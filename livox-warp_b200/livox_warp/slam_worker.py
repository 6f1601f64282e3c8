"""Odometry on its own thread and CUDA streams, for a render (or capture) thread that must not wait on it
(slam_worker.py, OdomWorker :100-338).

    caller thread (its current stream)                 worker thread (stream "odom")
    staged batch ──copy on stream "odom-in"──> input slot ──> frame cut, deskew, registration, keyframe insert
    frame slots <──copy on stream "odom-out"── deskewed frame points (on_frame, when a frame's pose is final)

The interface is the reference's: submit() hands over a staged batch, poll() returns FrameResults, reset(),
restart_clock(), configure(), status(), release_consumed() and close(); results carry a generation, and reset() or
restart_clock() drop whatever belongs to an older one. Hand-overs are own-or-drop: a full input queue, no free input
slot or no free output slot drops the item and counts it; poses always get through.

How it maps onto the device: the reference's worker exists because its registration reads back a 6x6 system on
every Gauss-Newton iteration; here a frame's whole registration is device work queued by one call, so the worker
thread spends its time waiting on its stream and the caller's stream never waits on the odometry's kernels. Batches
and frames cross between streams as copies into preallocated device slots, ordered by CUDA events: the consumer
stream waits for the copy's event, and the producer's next write to the source waits for the same event. Nothing
is allocated after construction.

Control plane: batches and commands (reset, restart, configure) travel in two deques under one condition variable.
Every batch carries its submission number, every command the number of batches submitted before it; the worker
runs a command as soon as no earlier batch is waiting, so commands and batches take effect in the order the caller
issued them. A new generation (reset, restart) releases the waiting batches of the old one at once.
"""

from __future__ import annotations

import collections
import sys
import threading
import time
import traceback
from dataclasses import dataclass, field

import numpy as np
import torch

from .gpu import Pipeline
from .odom import Odometry


class _Slots:
    """A fixed set of device buffer slots of the same shapes; take() gives a free slot index or None."""

    def __init__(self, n: int, shapes, dtypes, device):
        self.bufs = [[torch.zeros(s, dtype=dt, device=device) for s, dt in zip(shapes, dtypes)] for _ in range(n)]
        self._free = list(range(n - 1, -1, -1))
        self._lock = threading.Lock()

    def take(self) -> int | None:
        with self._lock:
            return self._free.pop() if self._free else None

    def give(self, i: int):
        with self._lock:
            self._free.append(i)

    @property
    def free_slots(self) -> int:
        with self._lock:
            return len(self._free)


class _Snap:
    """Rows [:n] of a slot, valid once `event` has completed; release() returns the slot."""

    def __init__(self, slots: _Slots, i: int, n: int, event: torch.cuda.Event):
        self._slots, self._i, self.n, self.event = slots, i, n, event
        self.arrays = [b[:n] for b in slots.bufs[i]]

    def wait(self, stream: torch.cuda.Stream):
        stream.wait_event(self.event)

    def release(self):
        if self._slots is not None:
            self._slots.give(self._i)
            self._slots = None


@dataclass
class FrameResult:
    gen: int
    k: int  # frame id
    T: np.ndarray  # sensor-to-world at mid-frame
    xi: np.ndarray  # body-frame motion over the frame (rho, theta)
    m: int  # points in the frame
    snaps: list | None  # [xyz (x, y, z), attr, t, frame] of the deskewed frame (device tensors), or None if dropped
    stats: dict = field(default_factory=dict)

    def arrays(self):
        return list(self.snaps) if self.snaps else []

    def release(self):
        if self._snap is not None:
            self._snap.release()
            self._snap = None
        self.snaps = None

    _snap: _Snap | None = None


@dataclass
class _Batch:
    seq: int  # submission number
    gen: int
    epoch: int
    snap: _Snap
    n: int
    t_min: float
    t_max: float


@dataclass
class _Command:
    after: int  # batches submitted before it: it runs once those have been taken
    kind: str  # "reset", "restart" or "configure"
    gen: int
    arg: object = None


class OdomWorker:
    """Runs an Odometry on its own thread and streams: the caller submits batches and polls FrameResults.

    in_slots batches can be in flight at once (each up to in_cap points); out_slots finished frames can wait for
    the caller (each up to frame_cap points)."""

    def __init__(self, pipe: Pipeline, device=None, max_batches: int = 120, out_slots: int = 8,
                 frame_cap: int = 1 << 18, in_slots: int = 32, in_cap: int = 1 << 16, reg_slots: int = 1 << 21):
        self.pipe = pipe
        d = torch.device(device) if device is not None else torch.device(pipe.device)
        if d.index is None:
            d = torch.device("cuda", torch.cuda.current_device())
        self.device = d
        with torch.cuda.device(d):
            self.s_in = torch.cuda.Stream(d)
            self.s_odom = torch.cuda.Stream(d)
            self.s_out = torch.cuda.Stream(d)
        self.odom = Odometry(pipe, d, reg_slots=reg_slots, frame_cap=frame_cap, stream=self.s_odom)
        self.in_cap = int(in_cap)
        self.in_pool = _Slots(in_slots, [(in_cap, 3), (in_cap,), (in_cap,)],
                              [torch.float32, torch.int32, torch.float32], d)
        self.out_pool = _Slots(out_slots, [(frame_cap, 3), (frame_cap,), (frame_cap,), (frame_cap,)],
                               [torch.float32, torch.int32, torch.float32, torch.int32], d)
        torch.cuda.synchronize(d)
        self.max_batches = max_batches
        self.gen = 0  # the caller's generation
        self._worker_gen = 0  # the generation the worker thread is on (written by that thread only)
        # work for the worker thread, guarded by _cv: batches and commands, ordered by submission number
        self._cv = threading.Condition()
        self._batches: collections.deque[_Batch] = collections.deque()
        self._commands: collections.deque[_Command] = collections.deque()
        self._submitted = 0
        self._running = 0  # batches taken by the worker and not yet finished
        self._stopping = False
        # finished frames for the caller
        self._ready: collections.deque[FrameResult] = collections.deque()
        self._ready_lock = threading.Lock()
        self._lock = threading.Lock()  # counters
        self.drops = {"input_full": 0, "input_own": 0, "output_pool": 0, "stale": 0, "error": 0}
        self.processed = 0
        self.frames = 0
        self.last_error = ""
        self.busy_ms = 0.0  # running average of worker time per batch
        self._consumed: list[FrameResult] = []
        self._closed = False
        self._thread = threading.Thread(target=self._serve, name="livox-odometry", daemon=True)
        self._thread.start()

    def _count(self, key: str, by: int = 1):
        with self._lock:
            self.drops[key] += by

    # ---- caller thread ----------------------------------------------------------------------------------

    def submit(self, sx, sa, st, n: int, t_min: float, t_max: float, epoch: int = 0) -> bool:
        """Hand one staged batch (device xyz [>=n, 3], attr, t, as Pipeline.stage returns them) to the worker.
        False = dropped (counted)."""
        if n <= 0:
            return True
        with self._cv:
            waiting = len(self._batches) + self._running
        if waiting >= self.max_batches:
            self._count("input_full")
            return False
        i = self.in_pool.take() if n <= self.in_cap else None
        if i is None:
            self._count("input_own")
            return False
        caller = torch.cuda.current_stream(self.device)
        ev = torch.cuda.Event()
        slot = self.in_pool.bufs[i]
        self.s_in.wait_stream(caller)  # the copy reads what the caller's stream staged
        with torch.cuda.stream(self.s_in):
            for dst, src in zip(slot, (sx[:n, :3], sa[:n], st[:n])):
                dst[:n].copy_(src, non_blocking=True)
            ev.record(self.s_in)
        caller.wait_event(ev)  # the caller's next write to its staging buffers waits for this copy
        with self._cv:
            self._batches.append(_Batch(self._submitted, self.gen, int(epoch), _Snap(self.in_pool, i, n, ev), n,
                                        float(t_min), float(t_max)))
            self._submitted += 1
            self._cv.notify()
        return True

    def _command(self, kind: str, arg=None, new_generation: bool = False):
        stale: list[_Batch] = []
        with self._cv:
            if new_generation:
                self.gen += 1
                stale = [b for b in self._batches if b.gen != self.gen]
                self._batches = collections.deque(b for b in self._batches if b.gen == self.gen)
            self._commands.append(_Command(self._submitted, kind, self.gen, arg))
            self._cv.notify()
        for b in stale:  # the old generation's batches give their slots back now
            b.snap.release()
        if stale:
            self._count("stale", len(stale))
        if new_generation:
            self._take_ready(self.gen)

    def reset(self, T0: np.ndarray):
        """Forget map and trajectory; the next frame is posed at T0. Batches and results of the old generation are
        discarded."""
        self._command("reset", np.array(T0, dtype=np.float64), new_generation=True)

    def restart_clock(self):
        """The clock restarted: keep the map and pose, restart frame counting at rest; the old clock's batches and
        results are discarded."""
        self._command("restart", new_generation=True)

    def configure(self, **params):
        """Set Odometry tuning attributes between batches; an unknown name raises AttributeError here."""
        for name in params:
            if not isinstance(getattr(self.odom, name, None), (int, float, str)):
                raise AttributeError(f"Odometry has no tuning attribute {name!r}")
        self._command("configure", dict(params))

    def _take_ready(self, gen: int) -> list[FrameResult]:
        """The finished frames of generation `gen`; the others are released and counted stale."""
        with self._ready_lock:
            items = list(self._ready)
            self._ready.clear()
        keep = [r for r in items if r.gen == gen]
        for r in items:
            if r.gen != gen:
                r.release()
        if len(keep) != len(items):
            self._count("stale", len(items) - len(keep))
        return keep

    def poll(self) -> list[FrameResult]:
        """Finished frames of the current generation; their arrays are ready for the caller's current stream. Call
        release_consumed() once that stream no longer reads them."""
        caller = torch.cuda.current_stream(self.device)
        out = self._take_ready(self.gen)
        for r in out:
            if r._snap is not None:
                r._snap.wait(caller)
        with self._lock:
            self.frames += len(out)
        self._consumed.extend(out)
        return out

    def release_consumed(self):
        """Return the polled frames' slots (after the caller's stream has passed the kernels that read them)."""
        for r in self._consumed:
            r.release()
        self._consumed.clear()

    def status(self) -> dict:
        with self._cv:
            pending = len(self._batches) + self._running
        with self._lock:
            return {"pending": pending, "processed": self.processed, "frames": self.frames,
                    "drops": dict(self.drops), "busy_ms": round(self.busy_ms, 2), "last_error": self.last_error,
                    "pool_free": min(self.in_pool.free_slots, self.out_pool.free_slots)}

    def close(self):
        if self._closed:
            return
        self._closed = True
        with self._cv:
            self.gen += 1
            stale = list(self._batches)
            self._batches.clear()
            self._stopping = True  # the commands already issued still run, then the thread ends
            self._cv.notify()
        for b in stale:
            b.snap.release()
        self._thread.join(timeout=10.0)
        self._take_ready(self.gen)
        self.release_consumed()
        if self._thread.is_alive():
            print("OdomWorker.close: the odometry thread did not stop", file=sys.stderr)

    # ---- worker thread ----------------------------------------------------------------------------------

    def _next(self):
        """Block until there is work: the next command when no earlier batch waits, else the next batch; None once
        close() has been called and the commands issued before it have run."""
        with self._cv:
            self._cv.wait_for(lambda: self._stopping or self._batches or self._commands)
            if self._commands and (not self._batches or self._commands[0].after <= self._batches[0].seq):
                return self._commands.popleft()
            if self._stopping:
                return None
            self._running += 1
            return self._batches.popleft()

    def _serve(self):
        torch.cuda.set_device(self.device)
        while (item := self._next()) is not None:
            try:
                if isinstance(item, _Batch):
                    self._batch(item)
                else:
                    self._apply(item)
            except Exception as e:  # one bad batch or command must not stop the worker
                with self._lock:
                    self.drops["error"] += 1
                    self.last_error = f"{type(e).__name__}: {e}"
                traceback.print_exc()

    def _apply(self, c: _Command):
        if c.kind == "configure":
            for name, value in c.arg.items():
                setattr(self.odom, name, value)
            return
        self._worker_gen = c.gen
        if c.kind == "reset":
            self.odom.reset(c.arg)
            self.odom.synchronize()
        else:
            self.odom.restart_clock()

    def _batch(self, item: _Batch):
        try:
            if item.gen != self._worker_gen:
                self._count("stale")
                return
            t0 = time.perf_counter()
            s = self.s_odom
            item.snap.wait(s)
            sx, sa, st = item.snap.arrays
            self.odom.epoch = item.epoch
            with torch.cuda.stream(s):
                self.odom.push(sx, sa, st, item.n, item.t_min, item.t_max, self._on_frame)
            s.synchronize()  # the odometry's reads of the input slot are done before it is reused
            dt = (time.perf_counter() - t0) * 1e3
            with self._lock:
                self.processed += 1
                self.busy_ms = dt if self.processed == 1 else 0.9 * self.busy_ms + 0.1 * dt
        finally:
            item.snap.release()
            with self._cv:
                self._running -= 1

    def _on_frame(self, k, T, fx, fa, ft, ff, m):
        """On the worker thread when a frame's pose is final: copy its points out for the caller."""
        o = self.odom
        st = o.read_state()
        xi = np.array(st.xi, dtype=np.float32)
        snap = None
        i = self.out_pool.take() if m <= o.frame_cap else None
        if i is None:
            self._count("output_pool")
        else:
            ev = torch.cuda.Event()
            slot = self.out_pool.bufs[i]
            self.s_out.wait_stream(self.s_odom)
            with torch.cuda.stream(self.s_out):
                for dst, src in zip(slot, (fx, fa, ft, ff)):
                    dst[:m].copy_(src[:m], non_blocking=True)
                ev.record(self.s_out)
            self.s_odom.wait_event(ev)  # the next frame's writes to fx .. ff wait for this copy
            snap = _Snap(self.out_pool, i, m, ev)
        r = FrameResult(self._worker_gen, int(k), np.array(T, dtype=np.float64), xi, int(m),
                        snap.arrays if snap else None, dict(o.stats))
        r._snap = snap
        with self._ready_lock:
            self._ready.append(r)
