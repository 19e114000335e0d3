"""shz_totals_noalloc: the conservation totals of a caller-owned device state with no allocation.

It serves callers that cannot let a library allocate device memory (a host keeping all GPU memory
in its own pool or fixed arena, or a binding handed buffers by another runtime). The GPU test
checks, through the C ABI, that two calls in a row give the totals of the existing entry point
(shz_diagnostics on a handle) within the tolerance the diagnostics tests use (1e-12 relative for
the compensated float64 sums, exact for the Mach maximum and the floored count). This file sorts
last so that a run stopping at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from shaderous_b200 import Config, Problem, Sim, _abi


def test_refuses_states_beyond_the_static_maximum():
    lib = _abi.load()
    cfg = Config(n=(1024, 512, 512)).to_c()  # 268M cells: twice the maximum
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    rc = lib.shz_totals_noalloc(C.byref(cfg), fake, fake, fake, None)
    assert rc == _abi.SHZ_E_CONFIG
    assert b"exceed" in lib.shz_totals_noalloc_error()
    assert _abi.SHZ_TOTALS_MAX_BLOCKS * _abi.SHZ_TOTALS_CELLS_PER_BLOCK == 512 ** 3


@pytest.mark.gpu
def test_noalloc_totals_match_handle_diagnostics_twice():
    import torch

    lib = _abi.load()
    n = 48
    cfg = Config(n=(n, n + 8, n - 8), gamma=1.4, recon="koren")
    with Sim(cfg) as s:
        s.reset(Problem("gauss", a=(1.5, 0.02, 1.0, 0.5, 0.1, 1.0, 0.01)))
        s.run(steps=5)
        d = s.diagnostics()
        s.sync()
        u1, u2 = s.state_device()
        want = np.array([d.mass, *d.momentum, d.e_kin, d.e_int, d.e_tot, d.floored, d.max_mach])
        c = cfg.to_c()
        for call in range(2):
            out = torch.full((_abi.SHZ_DIAG_VALUES,), float("nan"), dtype=torch.float64, device="cuda:0")
            torch.cuda.synchronize()
            rc = lib.shz_totals_noalloc(C.byref(c), C.c_void_p(u1), C.c_void_p(u2), C.c_void_p(out.data_ptr()), None)
            assert rc == 0, lib.shz_totals_noalloc_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.isfinite(got).all(), (call, got)
            np.testing.assert_allclose(got[:7], want[:7], rtol=1e-12, atol=1e-12 * abs(want[0]), err_msg=f"call {call}")
            assert got[7] == want[7] and got[8] == want[8], (call, got, want)
