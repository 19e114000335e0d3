"""The command-line runner on the library: the reference's headless `shaderous run / sweep /
describe` (tools/headless/cli.mjs, flags.mjs) for the problems and outputs this library has.

    python -m shaderous_b200 run "problem=sedov&dim=3&n=128" --until 0.02 --every 0.005 --out runs/sedov
    python -m shaderous_b200 run --problem kelvin-helmholtz --dim 2 --n 512 --set limiter=mc --steps 500
    python -m shaderous_b200 run "problem=sedov&dim=3&n=128&amr=4" --until 0.01
    python -m shaderous_b200 sweep --problem sod --n 512 --vary gamma=1.4,1.667 --until 0.2
    python -m shaderous_b200 describe [problem]

Outputs, as the reference's runner writes them: `diag.jsonl` (one line of diagnostics per output
time, at the start, every --every of simulated time and at the end) and `manifest.json` (the
setup, the outputs). With --athdf, each output also writes the run as an Athena++ HDF5 snapshot
NNNN-tT.athdf (src/io/athdf.ts; --gzip 1-9 compresses the cells), and --from FILE.athdf starts
the run from such a file (capture.ts restartFrom: its time, steps and gas, on a uniform grid or
on blocks). With --state, each output writes the raw state as NNNN-tT-state.npz (u1, u2 float32
arrays; uniform grids). Screenshots, slices and movies need the reference's renderer and are not
written.
"""
from __future__ import annotations

import argparse
import itertools
import json
import math
import sys
import time
from pathlib import Path
from urllib.parse import parse_qsl, urlencode

# Presets: problem kind, parameters, box (side), boundaries (lo, hi), gamma, end time, limiter.
# The parameters follow include/shaderous_b200.h SHZ_PROB_*.
PRESETS = {
    "sod": {"kind": "sod", "a": (1.0, 0.0, 1.0, 0.125, 0.0, 0.1), "box": 1.0, "bc": 1, "gamma": 1.4, "t_end": 0.2,
            "limiter": "minmod", "doc": "shock tube along x: (1, 0, 1) | (0.125, 0, 0.1), outflow"},
    "kelvin-helmholtz": {"kind": "kh", "a": (2.0, 1.0, 0.5, 2.5, 0.01, 1e-3), "box": 1.0, "bc": 0, "gamma": 1.4,
                         "t_end": 2.0, "limiter": "mc", "doc": "dense slab |y| < 1/4 at +0.5 through light gas at -0.5, periodic"},
    "sedov": {"kind": "sedov", "a": (1.0, 1e-5, 1.0, 3.5), "box": 1.0, "bc": 1, "gamma": 5.0 / 3.0, "t_end": 0.06,
              "limiter": "koren", "doc": "point blast, E = 1 within 3.5 cells of the centre, outflow"},
    "taylor-green": {"kind": "tgv", "a": (1.0, 100.0, 1.0), "box": 2.0 * math.pi, "bc": 0, "gamma": 5.0 / 3.0,
                     "t_end": 1.0, "limiter": "ppm", "doc": "3D Taylor-Green vortex on [0, 2 pi]^3, p0 = 100, periodic"},
    "blast": {"kind": "blast", "a": (1.0, 10.0, 1.0, 0.1, 0.1), "box": 1.0, "bc": 1, "gamma": 1.4, "t_end": 0.1,
              "limiter": "koren", "doc": "pressure sphere of radius 0.1, p 10 in 0.1, outflow"},
    "advection": {"kind": "advect", "a": (1.0, 0.5, 1.0, 0.0, 0.0, 1.0), "box": 1.0, "bc": 0, "gamma": 1.4, "t_end": 1.0,
                  "limiter": "koren", "doc": "smooth density wave carried across the periodic box"},
}
ALIASES = {"kh": "kelvin-helmholtz", "tgv": "taylor-green", "advect": "advection"}
NUMERIC = {"gamma", "cfl", "rho_floor", "p_floor", "eta_dual", "shock_thresh", "box", "t_end", "refine_hi", "refine_lo"}
INTEGER = {"dim", "n", "amr", "seed", "signal_dims", "regrid_every", "cap", "bc", "tbins"}


def parse_setup(query: str | None, ns) -> dict:
    """The setup from a query string (or link), the --problem/--dim/--n/--amr flags and --set."""
    keys: dict = {}
    if query:
        q = query.split("?", 1)[1] if "?" in query else query
        keys.update(dict(parse_qsl(q, keep_blank_values=True)))
    for k in ("problem", "dim", "n", "amr"):
        v = getattr(ns, k, None)
        if v is not None:
            keys[k] = v
    for kv in ns.set or []:
        if "=" not in kv or kv.startswith("="):
            raise SystemExit(f"error: --set takes KEY=VALUE, not {kv!r}")
        k, v = kv.split("=", 1)
        keys[k] = v
    name = ALIASES.get(str(keys.get("problem", "sod")), str(keys.get("problem", "sod")))
    if name not in PRESETS:
        raise SystemExit(f"error: unknown problem {name!r}; known: {', '.join(PRESETS)}")
    setup = {"problem": name}
    for k, v in keys.items():
        if k == "problem":
            continue
        if k in INTEGER:
            setup[k] = int(v)
        elif k in NUMERIC:
            setup[k] = float(v)
        else:
            setup[k] = v
    setup.setdefault("dim", 3 if name == "taylor-green" else 2 if name == "kelvin-helmholtz" else 1 if name == "sod" else 3)
    setup.setdefault("n", 128)
    return setup


def build(setup: dict):
    """(handle class, config, problem, end time) of a setup."""
    from .amr import AmrConfig, AmrSim
    from .sim import Config, Problem, Sim

    pre = PRESETS[setup["problem"]]
    dim, n = int(setup["dim"]), int(setup["n"])
    box = float(setup.get("box", pre["box"]))
    bc = int(setup.get("bc", pre["bc"]))
    limiter = str(setup.get("limiter", pre["limiter"]))
    cfg = Config(n=(n, n if dim >= 2 else 1, n if dim == 3 else 1), dx=box / n,
                 gamma=float(setup.get("gamma", pre["gamma"])), bc_lo=(bc,) * dim + (0,) * (3 - dim),
                 bc_hi=(bc,) * dim + (0,) * (3 - dim), cfl=float(setup.get("cfl", 0.8)), recon=limiter,
                 riemann=str(setup.get("riemann", "hllc")),
                 p_floor=float(setup.get("p_floor", 1e-12)), rho_floor=float(setup.get("rho_floor", 1e-10)),
                 isentropic=str(setup.get("isentropic", "1")) not in ("0", "false"))
    prob = Problem(pre["kind"], a=pre["a"], seed=int(setup.get("seed", 0)))
    t_end = float(setup.get("t_end", pre["t_end"]))
    levels = int(setup.get("amr", 0))
    if levels > 0:
        if dim < 2 or n % 16:
            raise SystemExit("error: an adaptive run needs dim 2 or 3 and n a multiple of 16 (the level-0 grid)")
        acfg = AmrConfig(hydro=cfg, ndim=dim, nr=n // 16, max_level=levels - 1, cap=int(setup.get("cap", 26000)),
                         box=box, refine_hi=float(setup.get("refine_hi", 0.1)),
                         refine_lo=float(setup.get("refine_lo", 0.05)), regrid_every=int(setup.get("regrid_every", 8)),
                         time_bins=int(setup.get("tbins", 0)))
        return AmrSim, acfg, prob, t_end
    return Sim, cfg, prob, t_end


def _diag_record(sim, wall: float) -> dict:
    d = sim.diagnostics_ext()
    t = d.totals
    return {"t": t.t, "dt": t.dt, "steps": t.steps, "wall": wall, "mass": t.mass, "momentum": list(t.momentum),
            "eKin": t.e_kin, "eInt": t.e_int, "eTot": t.e_tot, "maxMach": t.max_mach, "floored": t.floored,
            "com": list(d.com), "ranges": [list(d.ranges[k]) for k in ("rho", "temperature", "scalar", "pressure", "speed")]}


def run_one(setup: dict, ns, out: Path, log) -> dict:
    """One run: outputs at the start, every ns.every of simulated time and at the end."""
    import numpy as np

    cls, cfg, prob, t_end = build(setup)
    until = ns.until if ns.until is not None else (None if ns.steps is not None else t_end)
    out.mkdir(parents=True, exist_ok=True)
    manifest = {"setup": setup, "until": until, "steps": ns.steps, "every": ns.every, "outputs": []}
    t0 = time.perf_counter()
    with cls(cfg) as sim, open(out / "diag.jsonl", "w") as diag:
        sim.reset(prob)
        if getattr(ns, "from_file", None):
            from .athdf import read_athdf, restart

            restart(sim, read_athdf(ns.from_file))
            manifest["from"] = str(ns.from_file)

        def output(k: int):
            rec = _diag_record(sim, time.perf_counter() - t0)
            diag.write(json.dumps(rec) + "\n")
            diag.flush()
            entry = {"index": k, "t": rec["t"], "steps": rec["steps"]}
            if getattr(ns, "athdf", False):
                from .athdf import capture, write_athdf

                name = f"{k:04d}-t{rec['t']:.6g}.athdf"
                meta = {"program": "shaderous", "build": "b200", "query": urlencode({k2: str(v) for k2, v in setup.items()})}
                write_athdf(capture(sim, meta), out / name, gzip=getattr(ns, "gzip", 0) or 0)
                entry["athdf"] = name
            if ns.state and hasattr(sim, "read_state"):
                u1, u2 = sim.read_state()
                name = f"{k:04d}-t{rec['t']:.6g}-state.npz"
                np.savez(out / name, u1=u1, u2=u2)
                entry["state"] = name
            manifest["outputs"].append(entry)
            log(f"t = {rec['t']:.6g}  steps {rec['steps']}  mass {rec['mass']:.12g}  eTot {rec['eTot']:.12g}")

        output(0)
        k, taken = 1, 0
        stopped = "end"
        while True:
            target = until
            if ns.every and until is not None:
                target = min(until, ns.every * k)
            left_steps = None if ns.steps is None else ns.steps - taken
            if left_steps is not None and left_steps <= 0:
                stopped = "steps"
                break
            if ns.timeout and time.perf_counter() - t0 > ns.timeout:
                stopped = "timeout"
                break
            r = sim.run(steps=left_steps, until=target,
                        timeout_ms=(ns.timeout - (time.perf_counter() - t0)) * 1e3 if ns.timeout else None)
            taken += r.taken
            if r.stopped == "timeout":
                stopped = "timeout"
                break
            if until is not None and r.t >= until * (1 - 1e-12):
                stopped = "time"
                break
            if r.stopped == "steps" or r.taken == 0:
                stopped = r.stopped
                break
            output(k)
            k += 1
        output(k)
    manifest["stopped"] = stopped
    manifest["wall_seconds"] = time.perf_counter() - t0
    (out / "manifest.json").write_text(json.dumps(manifest, indent=1))
    return manifest


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m shaderous_b200", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("command", choices=["run", "sweep", "describe"])
    ap.add_argument("setup", nargs="?", help='a query string or link: "problem=sedov&dim=2&n=512"')
    ap.add_argument("--problem")
    ap.add_argument("--dim", type=int)
    ap.add_argument("--n", type=int)
    ap.add_argument("--amr", type=int, help="levels of the adaptive mesh (level 0 is the n grid)")
    ap.add_argument("--set", action="append", metavar="KEY=VALUE")
    ap.add_argument("--until", type=float)
    ap.add_argument("--steps", type=int)
    ap.add_argument("--every", type=float, help="outputs every this much simulated time")
    ap.add_argument("--timeout", type=float, help="give up after this many seconds of wall time")
    ap.add_argument("--out", help="output folder (default runs/<problem>-<date>)")
    ap.add_argument("--state", action="store_true", help="write the state at each output (.npz)")
    ap.add_argument("--athdf", action="store_true", help="write an Athena++ HDF5 snapshot at each output")
    ap.add_argument("--gzip", type=int, default=0, help="deflate level 1-9 for the snapshots' cells (0: none)")
    ap.add_argument("--from", dest="from_file", metavar="FILE", help="start from an .athdf snapshot")
    ap.add_argument("--vary", action="append", metavar="KEY=V1,V2,..")
    ap.add_argument("--quiet", action="store_true")
    ns = ap.parse_args(argv)
    log = (lambda m: None) if ns.quiet else (lambda m: print(m, file=sys.stderr))
    if ns.command == "describe":
        if ns.setup:
            name = ALIASES.get(ns.setup, ns.setup)
            if name not in PRESETS:
                raise SystemExit(f"error: unknown problem {ns.setup!r}")
            print(json.dumps({name: PRESETS[name]}, indent=1, default=str))
        else:
            print(json.dumps({k: v["doc"] for k, v in PRESETS.items()}, indent=1))
        return 0
    setup = parse_setup(ns.setup, ns)
    base = Path(ns.out) if ns.out else Path("runs") / f"{setup['problem']}-{time.strftime('%Y%m%d-%H%M%S')}"
    if ns.command == "run":
        m = run_one(setup, ns, base, log)
        print(json.dumps({"out": str(base), "stopped": m["stopped"], "outputs": len(m["outputs"])}))
        return 0
    if not ns.vary:
        raise SystemExit("error: sweep needs --vary KEY=V1,V2,..")
    axes = []
    for kv in ns.vary:
        k, vs = kv.split("=", 1)
        axes.append([(k, v) for v in vs.split(",")])
    results = []
    for combo in itertools.product(*axes):
        s = dict(setup)
        q = ns.__dict__.copy()
        s2 = parse_setup(None, argparse.Namespace(**{**q, "set": (ns.set or []) + [f"{k}={v}" for k, v in combo],
                                                     "problem": setup["problem"], "dim": setup["dim"], "n": setup["n"]}))
        s.update(s2)
        name = "-".join(f"{k}{v}" for k, v in combo)
        m = run_one(s, ns, base / name, log)
        results.append({"vary": dict(combo), "out": str(base / name), "stopped": m["stopped"]})
    print(json.dumps(results))
    return 0


if __name__ == "__main__":
    sys.exit(main())
