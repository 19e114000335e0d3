"""Serving over the C ABI: independent hydro requests resident in HBM, advanced together by the
block passes with continuous batching (shz_server_*), and the plain sequential loop beside it."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import load
from .sim import Config, Diagnostics, Problem, ShaderousError


@dataclass
class Request:
    ndim: int
    n: int
    steps: int
    problem: Problem
    gamma: float = 1.4
    bc: int = 0
    arrival: float = 0.0

    def to_c(self) -> _abi.shz_request:
        r = _abi.shz_request()
        r.ndim, r.n, r.steps, r.bc = self.ndim, self.n, self.steps, self.bc
        r.gamma, r.arrival = self.gamma, self.arrival
        r.problem = self.problem.to_c()
        return r

    @property
    def cells(self) -> int:
        return self.n ** self.ndim


@dataclass
class ServerConfig:
    hydro: Config = field(default_factory=lambda: Config(recon="koren", isentropic=True, cfl=0.4))
    budget_bytes: float = 8e9
    max_grids: int = 256
    round_steps: int = 8
    keep_states: bool = False
    direct_large: bool = True  # large requests run as uniform grids on streams of their own

    def to_c(self) -> _abi.shz_server_config:
        c = _abi.shz_server_config()
        c.hydro = self.hydro.to_c()
        c.budget_bytes = float(self.budget_bytes)
        c.max_grids, c.round_steps, c.keep_states = self.max_grids, self.round_steps, 1 if self.keep_states else 0
        c.direct_large = 1 if self.direct_large else 0
        return c


def _stats(st: _abi.shz_server_stats) -> dict:
    return {k: getattr(st, k) for k, _ in st._fields_}


def _array(reqs):
    arr = (_abi.shz_request * len(reqs))()
    for i, r in enumerate(reqs):
        arr[i] = r.to_c()
    return arr


class Server:
    def __init__(self, cfg: ServerConfig):
        self._lib = load()
        self.cfg = cfg
        h = C.c_void_p()
        rc = self._lib.shz_server_create(C.byref(cfg.to_c()), C.byref(h))
        if rc != 0:
            raise ShaderousError(rc, self._lib.shz_server_error(None).decode())
        self._h = h

    def _ok(self, rc):
        if rc != 0:
            raise ShaderousError(rc, self._lib.shz_server_error(self._h).decode())

    def destroy(self):
        if self._h:
            self._lib.shz_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def submit(self, req: Request) -> int:
        i = C.c_int64()
        self._ok(self._lib.shz_server_submit(self._h, C.byref(req.to_c()), C.byref(i)))
        return i.value

    def drain(self, max_rounds: int = 0):
        self._ok(self._lib.shz_server_drain(self._h, int(max_rounds)))

    def run_stream(self, reqs) -> dict:
        st = _abi.shz_server_stats()
        self._ok(self._lib.shz_server_run_stream(self._h, _array(reqs), len(reqs), C.byref(st)))
        return _stats(st)

    def cancel(self, rid: int) -> None:
        """Take request `rid` off the queue or the device; its result then raises SHZ_E_CANCELLED."""
        self._ok(self._lib.shz_server_cancel(self._h, int(rid)))

    def poll(self, rid: int) -> tuple[str, int]:
        """(status, steps taken) of request `rid`: status "queued", "running", "finished" or
        "cancelled"."""
        st, n = C.c_int32(), C.c_int64()
        self._ok(self._lib.shz_server_poll(self._h, int(rid), C.byref(st), C.byref(n)))
        return ("queued", "running", "finished", "cancelled")[st.value], n.value

    def result(self, rid: int) -> Diagnostics:
        d = _abi.shz_diag()
        self._ok(self._lib.shz_server_result(self._h, rid, C.byref(d)))
        return Diagnostics(d.t, d.dt, d.steps, d.mass, tuple(d.momentum), d.e_kin, d.e_int, d.e_tot, d.max_mach, d.floored)

    def state(self, rid: int, req: Request):
        u1 = np.zeros((req.cells, 4), np.float32)
        u2 = np.zeros((req.cells, 4), np.float32)
        self._ok(self._lib.shz_server_state(self._h, rid, u1.ctypes.data, u2.ctypes.data))
        return u1, u2


def plain_run_stream(cfg: ServerConfig, reqs) -> dict:
    lib = load()
    st = _abi.shz_server_stats()
    rc = lib.shz_plain_run_stream(C.byref(cfg.to_c()), _array(reqs), len(reqs), C.byref(st))
    if rc != 0:
        raise ShaderousError(rc, lib.shz_last_error(None).decode())
    return _stats(st)


def request_stream(count: int, seed: int = 2024, rate: float = 50.0, sizes2=(64, 1024), sizes3=(32, 256),
                   steps=(100, 2000)) -> list:
    """A seeded stream of Sod, Kelvin-Helmholtz and blast requests with Poisson arrivals: density
    ratio U[1, 10], pressure ratio log-U[1, 1000], gamma in {1.4, 5/3}, sizes log-uniform (multiples
    of 16), steps uniform."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        ndim = 2 if rng.random() < 0.5 else 3
        lo, hi = sizes2 if ndim == 2 else sizes3
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) / 16)) * 16
        n = max(16, min(hi, n))
        kind = ["sod", "kh", "blast"][int(rng.integers(3))]
        rr = float(rng.uniform(1, 10))
        pr = float(math.exp(rng.uniform(0, math.log(1000))))
        gamma = [1.4, 5.0 / 3.0][int(rng.integers(2))]
        if kind == "sod":
            prob, bc = Problem("sod", a=(rr, 0, pr, 1, 0, 1), axis=0), 1
        elif kind == "kh":
            prob, bc = Problem("kh", a=(rr, 1, 0.5, 2.5, 0.01, 1e-3), seed=int(rng.integers(1 << 62))), 0
        else:
            prob, bc = Problem("blast", a=(rr, pr, 1, 1, 0.15)), 1
        out.append(Request(ndim=ndim, n=n, steps=int(rng.integers(steps[0], steps[1] + 1)), problem=prob, gamma=gamma,
                           bc=bc, arrival=t))
    return out
