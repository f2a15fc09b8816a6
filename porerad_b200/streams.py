"""Independent calls on worker threads, each with its own CUDA stream on the caller's device.

libporerad releases the GIL while it waits for the device, and every call orders its work on
the calling thread's stream (``_lib.use_stream``); torch operations of a worker run on the same
stream.  Calls that are independent (seeds of a ray statistic, cells of a microstructure
library) then overlap on the GPU, and host work of one (NumPy fields, draws) overlaps the
device work of the others.
"""

from __future__ import annotations

import os
import threading
from concurrent.futures import ThreadPoolExecutor

from . import _lib

WORKERS = int(os.environ.get("PORERAD_WORKERS", "8"))
"""Worker threads (and streams); PORERAD_WORKERS overrides the default of 8."""

_pool = None
_pool_lock = threading.Lock()
_local = threading.local()


def _in_own_stream(device, fn, args, kwargs):
    import torch

    torch.cuda.set_device(device)  # the current device is per thread: the caller's, not device 0
    streams = getattr(_local, "streams", None)
    if streams is None:
        streams = _local.streams = {}
    if device not in streams:
        streams[device] = torch.cuda.Stream(device)
    stream = streams[device]
    with torch.cuda.stream(stream), _lib.use_stream(stream):
        try:
            return fn(*args, **kwargs)
        finally:
            stream.synchronize()  # results leave the worker complete


def run_concurrently(calls):
    """Results of calls [(fn, args, kwargs), ...] made on WORKERS threads with their own streams, in order."""

    global _pool
    import torch

    torch.cuda.synchronize()  # inputs were prepared on the caller's stream
    with _pool_lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(WORKERS, thread_name_prefix="porerad-worker")
    device = torch.cuda.current_device()
    futs = [_pool.submit(_in_own_stream, device, fn, args, kwargs) for fn, args, kwargs in calls]
    return [f.result() for f in futs]


def submit(fn, *args, **kwargs):
    """One call on a worker thread with its own stream; returns a Future.  Its inputs must be
    complete on the device (library calls that return host results are)."""

    global _pool
    import torch

    with _pool_lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(WORKERS, thread_name_prefix="porerad-worker")
    return _pool.submit(_in_own_stream, torch.cuda.current_device(), fn, args, kwargs)
