"""The launch-shape autotuner of the library's block and sweep kernels (``shz_tune_*``).

The first time a handle runs a tunable kernel for a (kernel, ndim, reconstruction, isentropic,
size class) key, the library times every candidate launch shape in place, inside one real step,
and keeps the fastest for the rest of the process. Candidates differ only in launch shape, so the
state is the same whichever wins.
"""
from __future__ import annotations

import ctypes as C

from . import _abi

KERNELS = {0: "uniform_sweep", 1: "amr_assemble", 2: "amr_sweep", 3: "amr_fine_flux", 4: "amr_assemble_bins"}


def enable(on: bool = True) -> None:
    """Turn the tuner on (the default) or off (every launch takes its default shape)."""
    _abi.load().shz_tune_enable(1 if on else 0)


def reset() -> None:
    """Forget every tuned choice."""
    _abi.load().shz_tune_reset()


def pin(kernel: str, variant: int | None, per_sm: int = 0) -> None:
    """Use this choice for every launch of a kernel instead of the tuned one; ``variant=None``
    unpins. AMR kernels ("amr_assemble", "amr_sweep", "amr_fine_flux", "amr_assemble_bins"): a
    variant and CTAs per SM. "uniform_sweep": variant 0 and ``per_sm`` = its depth (z planes a
    CTA marches in 3D; in 2D the rows it marches along y, 0 for the tile form)."""
    k = {v: n for n, v in KERNELS.items()}[kernel]
    rc = _abi.load().shz_tune_pin(k, -1 if variant is None else int(variant), int(per_sm))
    if rc != 0:
        raise ValueError(f"no choice {variant}, {per_sm} for {kernel}")


def entries() -> list[dict]:
    """The tuned choices: key, choice, and the mean times of the choice and of the default."""
    lib = _abi.load()
    n = C.c_int32()
    lib.shz_tune_entries(None, 0, C.byref(n))
    arr = (_abi.shz_tune_entry * max(n.value, 1))()
    lib.shz_tune_entries(arr, n.value, C.byref(n))
    out = []
    for e in arr[: n.value]:
        out.append({"kernel": KERNELS.get(e.kernel, str(e.kernel)), "ndim": e.ndim, "recon": e.recon,
                    "isentropic": e.isentropic, "size_class": e.size_class, "variant": e.variant,
                    "per_sm": e.per_sm, "tz": e.tz, "candidates": e.candidates, "ms": e.ms,
                    "default_ms": e.default_ms})
    return out
