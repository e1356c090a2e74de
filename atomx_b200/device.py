"""Device residency helpers: host<->device movement and a content-keyed cache
for the read-only basis arrays (grid nodes, weights, B-spline values, partial
matrices) so repeated calls on the same basis do not re-upload them."""
from __future__ import annotations

import hashlib
import threading
from collections import OrderedDict

import numpy as np
import torch

from . import _native

__all__ = ["as_device", "resident", "to_host", "is_device_tensor", "device", "wait_for"]

_cache: OrderedDict = OrderedDict()
_cache_lock = threading.Lock()
_CACHE_LIMIT = 256


def device() -> torch.device:
    _native.require_device()
    return torch.device("cuda", torch.cuda.current_device())


def is_device_tensor(x) -> bool:
    return isinstance(x, torch.Tensor) and x.is_cuda


def as_device(x, dtype=torch.float64, contiguous=True) -> torch.Tensor:
    """A contiguous device tensor view/copy of a numpy array or tensor."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device(), dtype=dtype) if (not x.is_cuda or x.dtype != dtype) else x
    else:
        arr = np.ascontiguousarray(np.asarray(x))
        if not arr.flags.writeable:
            arr = arr.copy()
        t = torch.from_numpy(arr).to(device=device(), dtype=dtype, non_blocking=False)
    return t.contiguous() if contiguous else t


def resident(x, dtype=torch.float64) -> torch.Tensor:
    """Device copy of a read-only host array, cached by content."""
    if isinstance(x, torch.Tensor) and x.is_cuda:
        return as_device(x, dtype)
    arr = np.ascontiguousarray(np.asarray(x))
    key = (arr.dtype.str, arr.shape, str(dtype), torch.cuda.current_device(),
           hashlib.blake2b(arr.tobytes(), digest_size=16).hexdigest())
    with _cache_lock:
        hit = _cache.get(key)
        if hit is not None:
            _cache.move_to_end(key)
            return hit
    t = as_device(arr, dtype)
    with _cache_lock:
        _cache[key] = t
        while len(_cache) > _CACHE_LIMIT:
            _cache.popitem(last=False)
    return t


def to_host(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu").numpy()


def wait_for(stream) -> None:
    """Block the calling host thread until ``stream`` has run the work queued
    on it so far, asleep in the driver rather than spinning: the wait goes
    through an event created with the blocking-sync flag.  Threads that spin
    while they wait use a core each; in a process with a CPU quota several of
    them can use it up and get the whole process throttled."""
    ev = torch.cuda.Event(blocking=True)
    ev.record(stream)
    ev.synchronize()
