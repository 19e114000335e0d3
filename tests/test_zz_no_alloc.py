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


def test_refuses_null_pointers_and_bad_device_index():
    lib = _abi.load()
    cfg = Config(n=(32, 32, 32)).to_c()
    fake = C.c_void_p(256)  # never dereferenced: every refusal here comes before a launch
    for args in [(None, fake, fake), (fake, None, fake), (fake, fake, None)]:
        rc = lib.shz_totals_noalloc(C.byref(cfg), *args, None)
        assert rc == _abi.SHZ_E_CONFIG
        assert b"null" in lib.shz_totals_noalloc_error()
    assert lib.shz_totals_noalloc(None, fake, fake, fake, None) == _abi.SHZ_E_CONFIG
    cfg.device = -1
    assert lib.shz_totals_noalloc(C.byref(cfg), fake, fake, fake, None) == _abi.SHZ_E_CONFIG
    assert b"device index -1" in lib.shz_totals_noalloc_error()


def test_error_message_is_per_thread():
    import threading

    lib = _abi.load()
    big = Config(n=(1024, 512, 512)).to_c()
    fake = C.c_void_p(256)
    assert lib.shz_totals_noalloc(C.byref(big), fake, fake, fake, None) == _abi.SHZ_E_CONFIG
    seen = {}

    def other():
        assert lib.shz_totals_noalloc(C.byref(big), None, fake, fake, None) == _abi.SHZ_E_CONFIG
        seen["other"] = lib.shz_totals_noalloc_error()

    t = threading.Thread(target=other)
    t.start()
    t.join()
    assert b"null" in seen["other"]
    assert b"exceed" in lib.shz_totals_noalloc_error()  # this thread's message is untouched


def _reference_totals(cfg):
    s = Sim(cfg)
    s.reset(Problem("gauss", a=(1.5, 0.02, 1.0, 0.5, 0.1, 1.0, 0.01)))
    s.run(steps=5)
    d = s.diagnostics()
    s.sync()
    return s, np.array([d.mass, *d.momentum, d.e_kin, d.e_int, d.e_tot, d.floored, d.max_mach])


def _check(got, want, tag):
    assert np.isfinite(got).all(), (tag, got)
    np.testing.assert_allclose(got[:7], want[:7], rtol=1e-12, atol=1e-12 * abs(want[0]), err_msg=tag)
    assert got[7] == want[7] and got[8] == want[8], (tag, got, want)


@pytest.mark.gpu
def test_noalloc_totals_match_handle_diagnostics_twice():
    import torch

    lib = _abi.load()
    n = 48
    cfg = Config(n=(n, n + 8, n - 8), gamma=1.4, recon="koren")
    s, want = _reference_totals(cfg)
    with s:
        u1, u2 = s.state_device()
        c = cfg.to_c()
        for call in range(2):
            out = torch.full((_abi.SHZ_DIAG_VALUES,), float("nan"), dtype=torch.float64, device="cuda:0")
            torch.cuda.synchronize()
            rc = lib.shz_totals_noalloc(C.byref(c), C.c_void_p(u1), C.c_void_p(u2), C.c_void_p(out.data_ptr()), None)
            assert rc == 0, lib.shz_totals_noalloc_error()
            torch.cuda.synchronize()
            _check(out.cpu().numpy(), want, f"call {call}")


@pytest.mark.gpu
def test_noalloc_totals_on_a_caller_stream_keep_the_current_device():
    import torch

    lib = _abi.load()
    cfg = Config(n=(40, 24, 16), gamma=5 / 3, recon="mc")
    s, want = _reference_totals(cfg)
    with s:
        u1, u2 = s.state_device()
        c = cfg.to_c()
        stream = torch.cuda.Stream(device="cuda:0")
        before = torch.cuda.current_device()
        for call in range(2):
            with torch.cuda.stream(stream):
                out = torch.full((_abi.SHZ_DIAG_VALUES,), float("nan"), dtype=torch.float64, device="cuda:0")
            stream.synchronize()
            rc = lib.shz_totals_noalloc(C.byref(c), C.c_void_p(u1), C.c_void_p(u2), C.c_void_p(out.data_ptr()),
                                        C.c_void_p(stream.cuda_stream))
            assert rc == 0, lib.shz_totals_noalloc_error()
            stream.synchronize()
            assert torch.cuda.current_device() == before
            _check(out.cpu().numpy(), want, f"stream call {call}")
        c.device = torch.cuda.device_count()  # one past the last device
        fake = C.c_void_p(256)
        assert lib.shz_totals_noalloc(C.byref(c), fake, fake, fake, None) == _abi.SHZ_E_CONFIG
        assert b"device(s) present" in lib.shz_totals_noalloc_error()
