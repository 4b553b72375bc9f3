"""Host tables of a chunked time loop, built in a helper process.

The per-step tables of the time loop (timeseries.build_series: the
reference's scalar chain of utci_process.py:917-1067 / solweig.py:1950-2122
and the per-patch increments of solweig.py:683-731, 1514-1635) depend on
the forcing, the site's height bound and its land-cover classes only.  They
cost a few milliseconds per site, mostly interpreter time over small torch
operations; built in the calling process they sit between the chunks'
launches, since the interpreter runs one of the two at a time.  A
spawn-started helper process builds them instead, while the caller launches
and the GPU runs, and sends each chunk's tables back as soon as they are
built.  It runs the same code on the same inputs, so the tables are the same
bits (torch's CPU kernels do not depend on the thread count at these sizes:
every vector is far below torch's parallel grain).

The helper is a separate interpreter started for this module alone
(``python -m``), so the caller's main script is never imported there.  A
job is one call's chunks in order; messages carry the job's number, so
the tables of an abandoned job are discarded, never taken for the next
one's.  A helper that dies raises in the caller; nothing falls back.
"""
from __future__ import annotations

import atexit
import itertools
import os
import subprocess
import sys
import threading
import traceback
from multiprocessing.connection import Connection


def _serve(inbox, outbox):
    import torch
    torch.set_num_threads(1)
    from . import timeseries as TS
    while True:
        try:
            job = inbox.recv()
        except EOFError:           # the caller's end closed: it exited
            return
        if job is None:
            return
        job_id, kw, starts, time_stop, chunk_steps, initial_scalars = job
        try:
            dc = TS.day_chain(kw["met_file"], kw["altitude"], kw["azimuth"], kw["zen"], kw["jday"],
                              kw["location"], starts[0] if starts else 0, time_stop)
            scalars = initial_scalars
            for t0 in starts:
                ser = TS.build_series(**kw, time_start=t0, time_stop=min(time_stop, t0 + chunk_steps),
                                      initial_scalars=scalars, day_chain=dc)
                scalars = ser.final
                outbox.send((job_id, "ok", ser))
        except BaseException:  # noqa: BLE001 -- reported to the caller, which raises
            outbox.send((job_id, "error", traceback.format_exc()))


class TableBuilder:
    """One helper process and its two pipes; jobs run one at a time.  The
    helper is started as ``python -m solweig_project_b200.hostwork`` (it
    imports this module only, not the caller's main script) and reads jobs
    from one inherited pipe, writing tables to the other."""

    def __init__(self):
        to_r, to_w = os.pipe()
        from_r, from_w = os.pipe()
        env = dict(os.environ)
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        env["PYTHONPATH"] = root + (os.pathsep + env["PYTHONPATH"] if env.get("PYTHONPATH") else "")
        try:
            self._proc = subprocess.Popen([sys.executable, "-m", __name__, str(to_r), str(from_w)],
                                          pass_fds=(to_r, from_w), env=env, stdin=subprocess.DEVNULL)
        finally:
            os.close(to_r)
            os.close(from_w)
        self._out = Connection(to_w, readable=False)
        self._in = Connection(from_r, writable=False)
        self._ids = itertools.count(1)
        self._lock = threading.Lock()

    def alive(self):
        return self._proc.poll() is None

    def close(self):
        if self.alive():
            try:
                self._out.send(None)
            except (BrokenPipeError, OSError):
                pass
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.terminate()
        self._out.close()
        self._in.close()

    def submit(self, kw, time_start, time_stop, chunk_steps, initial_scalars=None):
        """Start building the tables of steps [time_start, time_stop) in
        chunks of `chunk_steps`; returns a TableJob whose next() gives each
        chunk's Series in order.  `kw` holds build_series' other keyword
        arguments (the forcing, sun geometry, location, scale, amax, grid
        size, land-cover props and model parameters)."""
        starts = list(range(time_start, time_stop, chunk_steps))
        self._lock.acquire()
        try:
            job_id = next(self._ids)
            self._out.send((job_id, kw, starts, time_stop, chunk_steps, initial_scalars))
        except BaseException:
            self._lock.release()
            raise
        return TableJob(self, job_id, len(starts), (time_start, time_stop, chunk_steps))

    def _recv(self, job_id):
        while True:
            if not self._in.poll(0.5):
                if not self.alive():
                    raise RuntimeError("the host-table helper process exited")
                continue
            try:
                got_id, status, payload = self._in.recv()
            except EOFError:
                raise RuntimeError("the host-table helper process exited") from None
            if got_id != job_id:
                continue          # a message of an abandoned job
            if status == "error":
                raise RuntimeError("building the host tables failed in the helper process:\n" + payload)
            return payload


class TableJob:
    """The chunks of one submitted job, in order; finish() (or reading every
    chunk) releases the builder for the next job."""

    def __init__(self, builder, job_id, n, span=None):
        self._b, self._id, self._left = builder, job_id, n
        self._open = True
        self.span = span      # (time_start, time_stop, chunk_steps)

    def next(self):
        if self._left <= 0:
            raise StopIteration
        try:
            ser = self._b._recv(self._id)
        except BaseException:
            self.finish()
            raise
        self._left -= 1
        if self._left == 0:
            self.finish()
        return ser

    def finish(self):
        if self._open:
            self._open = False
            self._b._lock.release()


class LocalTables:
    """The same chunks built in this process when they are read (no helper
    process)."""

    def __init__(self, kw, time_start, time_stop, chunk_steps, initial_scalars=None):
        self.span = (time_start, time_stop, chunk_steps)
        self._kw, self._scalars, self._dc = kw, initial_scalars, None
        self._starts = list(range(time_start, time_stop, chunk_steps))

    def next(self):
        from . import timeseries as TS
        if not self._starts:
            raise StopIteration
        kw = self._kw
        t_start, time_stop, chunk_steps = self.span
        if self._dc is None:
            self._dc = TS.day_chain(kw["met_file"], kw["altitude"], kw["azimuth"], kw["zen"], kw["jday"],
                                    kw["location"], t_start, time_stop)
        t0 = self._starts.pop(0)
        ser = TS.build_series(**kw, time_start=t0, time_stop=min(time_stop, t0 + chunk_steps),
                              initial_scalars=self._scalars, day_chain=self._dc)
        self._scalars = ser.final
        return ser

    def finish(self):
        self._starts = []


_BUILDER = None
_BUILDER_LOCK = threading.Lock()


def builder() -> TableBuilder:
    """The process-wide helper, started on first use (and again if it died)."""
    global _BUILDER
    with _BUILDER_LOCK:
        if _BUILDER is None or not _BUILDER.alive():
            _BUILDER = TableBuilder()
        return _BUILDER


@atexit.register
def _shutdown():
    if _BUILDER is not None:
        _BUILDER.close()


if __name__ == "__main__":
    _serve(Connection(int(sys.argv[1]), writable=False), Connection(int(sys.argv[2]), readable=False))
