"""Serving front end over the hdd_server_* C ABI: resident domains, solve
requests from any thread, per-request latency.

The reference has no serving layer (its GPU demo solves one domain per
process); this mirrors the C interface one to one.  Solves on one domain and
on different domains run concurrently on the GPU; a request's result does not
depend on what else is in flight.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import HddError, hdd_options, hdd_result, hdd_server_options


def make_options(size, sub_size, vlevels=3, nVcycles=1, interior_smoothing=1, boundary_smoothing=3,
                 sigma_levels=3, sigma_smoothing=3, sigma_mg=1, **extra) -> hdd_options:
    """hdd_options from the reference's Test_Bench arguments (plus any hdd_options field)."""
    lib = _lib.load()
    o = hdd_options()
    lib.hdd_options_default(C.byref(o))
    for a in range(3):
        o.size[a] = int(size[a])
        o.sub_size[a] = int(sub_size[a])
    o.vlevels, o.nVcycles = vlevels, nVcycles
    o.interior_smoothing, o.boundary_smoothing = interior_smoothing, boundary_smoothing
    o.sigma_levels, o.sigma_smoothing, o.sigma_mg = sigma_levels, sigma_smoothing, sigma_mg
    for k, v in extra.items():
        setattr(o, k, v)
    return o


class SolveServer:
    def __init__(self, slots: int = 4, hbm_budget_bytes: int = 0, device: int = 0, setup_threads: int = 0,
                 batch: int = 0):
        self.lib = _lib.load()
        o = hdd_server_options()
        self.lib.hdd_server_options_default(C.byref(o))
        o.slots, o.hbm_budget_bytes, o.device, o.setup_threads = slots, hbm_budget_bytes, device, setup_threads
        o.batch = batch
        h = C.c_void_p()
        self._check(self.lib.hdd_server_create(C.byref(o), C.byref(h)))
        self.h = h
        self.sizes = {}

    def _check(self, st, domain=None):
        if st != 0:
            msg = (self.lib.hdd_status_string(st) or b"").decode()
            if domain is not None:
                buf = C.create_string_buffer(512)
                if self.lib.hdd_server_domain_error(self.h, domain, buf, 512) == 0 and buf.value:
                    msg = buf.value.decode()
            raise HddError(st, msg)

    def add_domain(self, flags: np.ndarray, options: hdd_options) -> int:
        flags = np.ascontiguousarray(flags, np.uint32)
        size = tuple(options.size)
        if flags.shape != size:
            raise HddError(1, f"flags shape {flags.shape} differs from options.size {size}")
        d = C.c_longlong()
        self._check(self.lib.hdd_server_add_domain(self.h, C.byref(options),
                                                   flags.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(d)))
        self.sizes[d.value] = size
        return d.value

    def wait_domain(self, domain: int, wait_ms: int = -1) -> bool:
        """True once resident, False while pending; raises if its setup failed."""
        st = self.lib.hdd_server_domain_status(self.h, domain, wait_ms)
        if st == 10:
            return False
        self._check(st, domain)
        return True

    def submit(self, domain: int, rhs: np.ndarray) -> int:
        rhs = np.ascontiguousarray(rhs, np.float32)
        if rhs.shape != self.sizes.get(domain):
            raise HddError(1, f"rhs shape {rhs.shape} differs from the domain's {self.sizes.get(domain)}")
        r = C.c_longlong()
        self._check(self.lib.hdd_server_submit(self.h, domain, rhs.ctypes.data_as(C.POINTER(C.c_float)),
                                               C.byref(r)))
        return r.value

    def poll(self, request: int, domain: int, wait_ms: int = -1, want_x: bool = True):
        """None while pending, else (status, result dict, x or None, latency_ms)."""
        res = hdd_result()
        lat = C.c_double()
        x = np.zeros(self.sizes[domain], np.float32) if want_x else None
        xp = x.ctypes.data_as(C.POINTER(C.c_float)) if want_x else None
        st = self.lib.hdd_server_poll(self.h, request, wait_ms, C.byref(res), xp, C.byref(lat))
        if st == 10:
            return None
        if st == 11:
            raise HddError(st, "unknown request")
        return st, {f: getattr(res, f) for f, _ in hdd_result._fields_}, x, lat.value

    def remove_domain(self, domain: int):
        self._check(self.lib.hdd_server_remove_domain(self.h, domain))
        self.sizes.pop(domain, None)

    def memory(self):
        r, b = C.c_longlong(), C.c_longlong()
        self._check(self.lib.hdd_server_memory(self.h, C.byref(r), C.byref(b)))
        return r.value, b.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.hdd_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
