"""Python face of the serving loop (include/picard_server.h).

A ``Server`` admits runs by HBM budget and runs them concurrently on the
device, each on its own CUDA stream driven by a native worker thread; the
Python side only submits requests and collects results.  The reference has no
serving layer (one `program picard` process per parameter set,
picard.f90:42-52 and 145-302); a request here carries the run's whole
parameter block.
"""
from __future__ import annotations

import ctypes as C

from . import capi
from .params import PicardParams


class Server:
    """``batched=False``: one worker thread and CUDA stream per slot, each run
    driven alone (picard_server_create).  ``batched=True``: continuous
    batching (picard_server_create_batched) -- up to ``slots`` admitted runs
    advanced together one iteration at a time, all their Jacobi sweeps in one
    launch per sweep, ``preparers`` threads building newly admitted runs."""

    def __init__(self, hbm_budget_bytes: int, slots: int, batched: bool = False, preparers: int = 2,
                 devices: "list[int] | None" = None):
        """``devices``: place runs over these device ordinals (one shard each,
        ``hbm_budget_bytes`` and ``slots`` per shard; picard_server_create_multi);
        None: the current device only."""
        self._lib = capi.lib()
        self._h = C.c_void_p()
        if devices is not None:
            arr = (C.c_int32 * len(devices))(*[int(d) for d in devices])
            capi.check(self._lib.picard_server_create_multi(arr, len(devices), int(hbm_budget_bytes), int(slots),
                                                            1 if batched else 0, int(preparers), C.byref(self._h)),
                       "picard_server_create_multi")
        elif batched:
            capi.check(self._lib.picard_server_create_batched(int(hbm_budget_bytes), int(slots), int(preparers),
                                                              C.byref(self._h)), "picard_server_create_batched")
        else:
            capi.check(self._lib.picard_server_create(int(hbm_budget_bytes), int(slots), C.byref(self._h)),
                       "picard_server_create")
        self.budget = int(hbm_budget_bytes)
        self.slots = int(slots)
        self.batched = bool(batched)

    def submit(self, rid: int, params: PicardParams, steps: int, layout: int = capi.LAYOUT_CELL32,
               solver: int = capi.SOLVER_F32_REFINE, arrival_ms: float = -1.0) -> None:
        """Queue a run; ``params`` must already be derived."""
        rq = capi.PicardRequest()
        rq.id = int(rid)
        rq.params = params
        rq.layout = layout
        rq.solver = solver
        rq.steps = int(steps)
        rq.arrival_ms = float(arrival_ms)
        capi.check(self._lib.picard_server_submit(self._h, C.byref(rq)), "picard_server_submit")

    def now_ms(self) -> float:
        t = C.c_double(0.0)
        capi.check(self._lib.picard_server_now_ms(self._h, C.byref(t)), "picard_server_now_ms")
        return t.value

    def poll(self, wait_all: bool = False, max_results: int = 4096) -> list[dict]:
        buf = (capi.PicardResult * max_results)()
        n = C.c_int32(0)
        capi.check(self._lib.picard_server_poll(self._h, buf, max_results, C.byref(n), 1 if wait_all else 0),
                   "picard_server_poll")
        return [buf[i].as_dict() for i in range(n.value)]

    def load(self) -> tuple[int, int, int]:
        """(runs in flight, runs queued, HBM bytes held by admitted runs)."""
        r, q, b = C.c_int32(0), C.c_int32(0), C.c_uint64(0)
        capi.check(self._lib.picard_server_load(self._h, C.byref(r), C.byref(q), C.byref(b)), "picard_server_load")
        return r.value, q.value, int(b.value)

    def close(self) -> None:
        if self._h:
            capi.check(self._lib.picard_server_destroy(self._h), "picard_server_destroy")
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
