"""The simulator as an MCP server (Model Context Protocol over stdio), the reference's
tools/headless/mcp.mjs for what this library has: an agent loads a setup, runs it, and reads the
gas back as tools. One simulation at a time, kept between calls.

    python -m shaderous_b200.mcp

Messages are JSON-RPC 2.0, one per line on stdin and stdout (mcp.mjs:322-337); logging goes to
stderr. Tools: describe, check_setup, load, run, state, diagnostics, stats, slice, probe, restart,
save_athdf, load_athdf, errors. The reference's screenshot, record, view and control tools drive its
renderer and page, which this library does not have (no graphics stack on this path); they are not
offered. A tool that fails answers with isError and the message, so the caller can correct its call
(mcp.mjs:305-309).
"""
from __future__ import annotations

import json
import math
import sys
import traceback
from pathlib import Path
from urllib.parse import urlencode

from . import cli

PROTOCOL = "2025-06-18"
VERSION = "0.1.0"
INSTRUCTIONS = (
    "Shaderous-B200 runs the compressible Euler equations (ideal gas) on one B200, on a uniform grid "
    "or an adaptive block mesh. These tools drive one simulation. Typical use: describe (pick a "
    "problem) -> load (a setup: problem, dim, n, amr and other keys, as a query string) -> run (to a "
    "time, landed on exactly, or a number of steps) -> diagnostics / stats / slice / probe for numbers "
    "-> save_athdf to keep the state. All values are in code units; positions are fractions of the "
    "box (0 to 1). A run stays where it stopped between calls; load starts from t = 0.")

VARIABLES = ("rho", "pressure", "vx", "vy", "vz", "speed", "scalar", "eint")


def _schema(props: dict, required=()) -> dict:
    return {"type": "object", "properties": props, "required": list(required)}


TOOL_DOCS = {
    "describe": ("The problems this library has (with `problem`: that preset's keys and defaults) and the "
                 "setup keys a load takes.",
                 _schema({"problem": {"type": "string"}})),
    "check_setup": ("Parse a setup (a query string such as \"problem=sedov&dim=3&n=128\") without loading it: "
                    "the keys as they would be used, or why it is refused.",
                    _schema({"setup": {"type": "string"}}, ["setup"])),
    "load": ("Load a setup and its initial conditions (t = 0). Keys: " + ", ".join(
        ["problem", "dim", "n", "amr", "box", "bc", "gamma", "cfl", "limiter", "riemann", "isentropic", "t_end",
         "rho_floor", "p_floor", "refine_hi", "refine_lo", "regrid_every", "cap", "tbins", "seed"]) + ".",
             _schema({"setup": {"type": "string"}}, ["setup"])),
    "run": ("Run the loaded simulation: to `until` (the last step shortened to land on it), or `steps` steps, "
            "or both; gives up after timeout_seconds (default 600) of wall time.",
            _schema({"until": {"type": "number"}, "steps": {"type": "integer"},
                     "timeout_seconds": {"type": "number"}})),
    "state": ("The loaded setup and its clock (t, dt, steps).", _schema({})),
    "diagnostics": ("Float64 totals (mass, momentum, kinetic, internal and total energy, floored cells, "
                    "largest Mach number), the centre of mass and the ranges of density, temperature, scalar, "
                    "pressure and speed.", _schema({})),
    "stats": ("The mesh: cells, and on the adaptive mesh its leaves per level; the kernels launched so far.",
              _schema({})),
    "slice": ("A slice of a variable (" + ", ".join(VARIABLES) + ") normal to `axis` (0, 1, 2) at fraction `pos`, "
              "sampled on res x res points: min, max, mean, and the values when res <= 64 or include_values; "
              "save_path writes .npy or .json.",
              _schema({"variable": {"type": "string"}, "axis": {"type": "integer"}, "pos": {"type": "number"},
                       "res": {"type": "integer"}, "include_values": {"type": "boolean"},
                       "save_path": {"type": "string"}}, ["variable"])),
    "probe": ("The gas at points (each [x, y, z] in fractions of the box): density, velocity, pressure, scalar "
              "of the cell that holds it.",
              _schema({"points": {"type": "array", "items": {"type": "array", "items": {"type": "number"}}}},
                      ["points"])),
    "restart": ("Load the same setup again from t = 0.", _schema({})),
    "save_athdf": ("Write the run as an Athena++ HDF5 snapshot (.athdf) at `path`.",
                   _schema({"path": {"type": "string"}, "gzip": {"type": "integer"}}, ["path"])),
    "load_athdf": ("Restart the loaded run from an .athdf snapshot: its time, steps and gas.",
                   _schema({"path": {"type": "string"}}, ["path"])),
    "errors": ("The errors of this session's tool calls, last first.", _schema({})),
}


class Session:
    """One simulation, kept between tool calls."""

    def __init__(self):
        self.sim = None
        self.setup = None
        self.query = ""
        self.error_log: list[str] = []

    # -- helpers -------------------------------------------------------------------------------
    def _need(self):
        if self.sim is None:
            raise ValueError("no run is loaded: call load first")
        return self.sim

    def _close(self):
        if self.sim is not None:
            self.sim.destroy()
            self.sim = None

    def _parse(self, query: str) -> dict:
        class NS:
            problem = dim = n = amr = None
            set = None

        try:
            return cli.parse_setup(query, NS())
        except SystemExit as e:  # parse_setup refuses with SystemExit("error: ...")
            raise ValueError(str(e).removeprefix("error: ")) from None

    @staticmethod
    def _build(s: dict):
        try:
            return cli.build(s)
        except SystemExit as e:  # build refuses with SystemExit("error: ...")
            raise ValueError(str(e).removeprefix("error: ")) from None

    def _clock(self) -> dict:
        t, dt, steps = self._need().clock()
        return {"t": t, "dt": dt, "steps": steps}

    def _cells(self):
        """The run as a snapshot (athdf.capture): every leaf's cells and primitives."""
        from .athdf import capture

        return capture(self._need(), {"program": "shaderous", "build": "b200", "query": self.query})

    # -- tools ---------------------------------------------------------------------------------
    def describe(self, problem: str | None = None):
        if problem:
            name = cli.ALIASES.get(problem, problem)
            if name not in cli.PRESETS:
                raise ValueError(f"no problem \"{problem}\": call describe without arguments for the list")
            p = dict(cli.PRESETS[name])
            p["a"] = list(p["a"])
            return {"id": name, **p}
        return {"problems": [{"id": k, "doc": v["doc"], "tEnd": v["t_end"], "limiter": v["limiter"]}
                             for k, v in cli.PRESETS.items()],
                "variables": list(VARIABLES),
                "limiters": ["minmod", "mc", "vanleer", "koren", "ppm"], "riemann": ["hllc", "hll"],
                "setupKeys": TOOL_DOCS["load"][0]}

    def check_setup(self, setup: str):
        s = self._parse(setup)
        cls, cfg, _, t_end = self._build(s)
        return {"setup": s, "grid": "adaptive" if cls.__name__ == "AmrSim" else "uniform", "tEnd": t_end}

    def load(self, setup: str):
        s = self._parse(setup)
        cls, cfg, prob, t_end = self._build(s)
        self._close()
        sim = cls(cfg)
        try:
            sim.reset(prob)
        except Exception:
            sim.destroy()
            raise
        self.sim, self.setup = sim, s
        self.query = urlencode({k: str(v) for k, v in s.items()})
        return {"loaded": s, "tEnd": t_end, **self._clock()}

    def run(self, until=None, steps=None, timeout_seconds=None):
        if until is None and steps is None:
            raise ValueError("run needs `until`, `steps`, or both")
        r = self._need().run(steps=steps, until=until, timeout_ms=1000.0 * (timeout_seconds or 600))
        return {"t": r.t, "dt": r.dt, "steps": r.steps, "taken": r.taken, "seconds": r.seconds,
                "stopped": r.stopped, "lastDt": r.last_dt}

    def state(self):
        return {"setup": self.setup, **self._clock()} if self.sim is not None else {"setup": None}

    def diagnostics(self):
        d = self._need().diagnostics_ext()
        t = d.totals
        return {"t": t.t, "dt": t.dt, "steps": t.steps, "mass": t.mass, "momentum": list(t.momentum),
                "eKin": t.e_kin, "eInt": t.e_int, "eTot": t.e_tot, "maxMach": t.max_mach, "floored": t.floored,
                "centerOfMass": list(d.com),
                "ranges": {k: list(d.ranges[k]) for k in ("rho", "temperature", "scalar", "pressure", "speed")}}

    def stats(self):
        sim = self._need()
        out = {"kernelLaunches": sim.kernel_launches}
        if hasattr(sim, "leaves"):
            import numpy as np

            _, levels, _ = sim.leaves()
            cb = 16 ** self.setup["dim"]
            out.update({"leaves": int(len(levels)), "cells": int(len(levels)) * cb,
                        "leavesPerLevel": np.bincount(levels).tolist()})
        else:
            n = self.setup["n"]
            out["cells"] = n ** self.setup["dim"]
        return out

    def _sample(self, points):
        """Primitives at points given as fractions of the box: (n, 6) rho, v, p, s of the cells that
        hold them (the finest leaf on the adaptive mesh; athdf.SnapshotSampler)."""
        import numpy as np

        from .athdf import SnapshotSampler

        snap = self._cells()
        smp = SnapshotSampler(snap)
        pts = np.asarray(points, np.float64).reshape(-1, 3)
        b, c = smp.lookup(pts[:, 0], pts[:, 1], pts[:, 2])
        o = b.astype(np.int64) * smp.cells + c
        d = snap.data
        cols = [d["rho"], d["vel1"], d["vel2"], d["vel3"], d["press"],
                d["r0"] if d.get("r0") is not None else np.zeros_like(d["rho"])]
        return np.stack([np.asarray(x).reshape(-1)[o] for x in cols], axis=1).astype(np.float64)

    def slice(self, variable, axis=2, pos=0.5, res=32, include_values=None, save_path=None):
        import numpy as np

        if variable not in VARIABLES:
            raise ValueError(f"variable must be one of {', '.join(VARIABLES)}")
        dim = self.setup["dim"] if self.setup else 3
        if not 0 <= axis < 3:
            raise ValueError("axis must be 0, 1 or 2")
        res = int(res)
        if not 1 <= res <= 2048:
            raise ValueError("res must be 1 to 2048")
        axes = [a for a in range(3) if a != axis][:2]
        g = (np.arange(res) + 0.5) / res
        pts = np.zeros((res * res, 3))
        pts[:, axes[0]] = np.tile(g, res)
        pts[:, axes[1]] = np.repeat(g, res)
        pts[:, axis] = pos
        w = self._sample(pts)
        rho, v, p, s = w[:, 0], w[:, 1:4], w[:, 4], w[:, 5]
        gamma = float(self.setup.get("gamma", cli.PRESETS[self.setup["problem"]]["gamma"]))
        vals = {"rho": rho, "pressure": p, "vx": v[:, 0], "vy": v[:, 1], "vz": v[:, 2],
                "speed": np.sqrt((v ** 2).sum(axis=1)), "scalar": s, "eint": p / (gamma - 1) / rho}[variable]
        vals = vals.astype(np.float32)
        out = {**self._clock(), "variable": variable, "axis": axis, "pos": pos, "res": res, "axes": axes,
               "min": float(vals.min()), "max": float(vals.max()), "mean": float(vals.mean())}
        if save_path:
            f = Path(save_path).resolve()
            f.parent.mkdir(parents=True, exist_ok=True)
            if f.suffix.lower() == ".npy":
                np.save(f, vals.reshape(res, res))
            else:
                f.write_text(json.dumps({**out, "values": vals.tolist()}) + "\n")
            out["saved"] = str(f)
            return out
        if include_values if include_values is not None else res <= 64:
            out["values"] = [[float(f"{x:.5g}") for x in row] for row in vals.reshape(res, res)]
        return out

    def probe(self, points):
        w = self._sample(points)
        return {**self._clock(),
                "points": [{"at": list(map(float, pt)), "rho": float(x[0]), "v": [float(x[1]), float(x[2]), float(x[3])],
                            "p": float(x[4]), "scalar": float(x[5])} for pt, x in zip(points, w)]}

    def restart(self):
        if self.setup is None:
            raise ValueError("no run is loaded: call load first")
        return self.load(self.query)

    def save_athdf(self, path, gzip=0):
        from .athdf import write_athdf

        snap = self._cells()
        f = Path(path).resolve()
        f.parent.mkdir(parents=True, exist_ok=True)
        write_athdf(snap, f, gzip=int(gzip or 0))
        return {"saved": str(f), "time": snap.time, "bytes": f.stat().st_size}

    def load_athdf(self, path):
        from .athdf import read_athdf, restart

        restart(self._need(), read_athdf(Path(path).resolve()))
        return {"restarted": str(Path(path).resolve()), **self._clock()}

    def errors(self):
        return {"errors": self.error_log[::-1]}


def _text(v) -> dict:
    def rnd(x):
        if isinstance(x, float) and math.isfinite(x) and not x.is_integer():
            return float(f"{x:.7g}")
        if isinstance(x, dict):
            return {k: rnd(y) for k, y in x.items()}
        if isinstance(x, (list, tuple)):
            return [rnd(y) for y in x]
        return x

    return {"content": [{"type": "text", "text": v if isinstance(v, str) else json.dumps(rnd(v), indent=1)}]}


class Server:
    """JSON-RPC 2.0 over lines (mcp.mjs:312-337)."""

    def __init__(self):
        self.session = Session()

    def handle(self, msg: dict) -> dict | None:
        mid, method, params = msg.get("id"), msg.get("method"), msg.get("params") or {}

        def reply(result):
            return None if mid is None else {"jsonrpc": "2.0", "id": mid, "result": result}

        def error(code, message):
            return None if mid is None else {"jsonrpc": "2.0", "id": mid, "error": {"code": code, "message": message}}

        if method == "initialize":
            return reply({"protocolVersion": params.get("protocolVersion", PROTOCOL), "capabilities": {"tools": {}},
                          "serverInfo": {"name": "shaderous-b200", "version": VERSION},
                          "instructions": INSTRUCTIONS})
        if method == "ping":
            return reply({})
        if method == "tools/list":
            return reply({"tools": [{"name": k, "description": d, "inputSchema": s} for k, (d, s) in TOOL_DOCS.items()]})
        if method == "tools/call":
            name = params.get("name")
            if name not in TOOL_DOCS:
                return error(-32602, f"unknown tool \"{name}\"")
            try:
                return reply(_text(getattr(self.session, name)(**(params.get("arguments") or {}))))
            except Exception as e:  # reported to the caller, which can correct its call
                msg_ = f"{type(e).__name__}: {e}" if not isinstance(e, ValueError) else str(e)
                self.session.error_log.append(f"{name}: {msg_}")
                return reply({"content": [{"type": "text", "text": f"Error: {msg_}"}], "isError": True})
        if isinstance(method, str) and method.startswith("notifications/"):
            return None
        return error(-32601, f"method not found: {method}")


def serve(inp=sys.stdin, out=sys.stdout, log=sys.stderr) -> None:
    srv = Server()
    print("[shaderous-b200-mcp] ready", file=log, flush=True)
    for line in inp:
        if not line.strip():
            continue
        try:
            msg = json.loads(line)
        except json.JSONDecodeError:
            out.write(json.dumps({"jsonrpc": "2.0", "id": None, "error": {"code": -32700, "message": "parse error"}}) + "\n")
            out.flush()
            continue
        try:
            r = srv.handle(msg)
        except Exception:
            traceback.print_exc(file=log)
            continue
        if r is not None:
            out.write(json.dumps(r) + "\n")
            out.flush()
    srv.session._close()


if __name__ == "__main__":
    serve()
