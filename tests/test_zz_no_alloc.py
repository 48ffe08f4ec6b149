"""fdtd_dft_noalloc: the device DFT for callers that must not allocate GPU memory.

Some hosts of this library cannot call cudaMalloc: their device memory is
owned by another component's pool or fixed budget, or they run the transform
in a loop where cudaMalloc/cudaFree, which can synchronise the whole device,
is not allowed.  For them the library stages the DFT through one fixed
device array instead of allocating.  This test calls that entry point through
the C ABI and checks it against the allocating fdtd_dft, twice in a row with
different sizes (the second call smaller, so left-over data from the first
would show), and checks that the device's free memory is the same before and
after a run of calls: no call keeps device memory.  (A buffer that a call
allocated and freed again before returning would not show there; the source
of the entry point calls no allocator.)  It lives in its own file, collected
last.
"""
import numpy as np
import pytest

from conftest import load_package

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402

pytestmark = pytest.mark.gpu


def _dft(fn, x, dt, f, shift):
    re, im = np.zeros(f.size), np.zeros(f.size)
    N.check(fn(N.dptr(x), x.size, dt, N.dptr(f), f.size, shift, N.dptr(re), N.dptr(im)))
    return re + 1j * im


def test_noalloc_dft_matches_allocating_dft_on_two_calls():
    L = N.lib()
    rng = np.random.default_rng(42)
    dt = 5.77e-13
    cases = [(np.ascontiguousarray(rng.standard_normal(7000)), np.linspace(2e7, 1e10, 500), 0.0),
             (np.ascontiguousarray(rng.standard_normal(1500)), np.linspace(1e9, 4e9, 301), -dt / 2)]
    for x, f, shift in cases:
        f = np.ascontiguousarray(f)
        got = _dft(L.fdtd_dft_noalloc, x, dt, f, shift)
        ref = _dft(L.fdtd_dft, x, dt, f, shift)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def _free_device_bytes() -> int:
    """cudaMemGetInfo of the current device, through the CUDA runtime the
    process already has loaded."""
    import torch
    free, _ = torch.cuda.mem_get_info(0)
    return int(free)


def test_noalloc_dft_keeps_no_device_memory():
    L = N.lib()
    rng = np.random.default_rng(7)
    dt = 5.77e-13
    x = np.ascontiguousarray(rng.standard_normal(4000))
    f = np.ascontiguousarray(np.linspace(1e9, 4e9, 301))
    _free_device_bytes()                         # the query's own first-use set-up
    _dft(L.fdtd_dft_noalloc, x, dt, f, 0.0)      # first call on the device: symbol set-up
    before = _free_device_bytes()
    for n, m in ((4000, 301), (32768, 4096), (10, 1), (7000, 500)):
        xs = np.ascontiguousarray(rng.standard_normal(n))
        fs = np.ascontiguousarray(np.linspace(1e8, 1e10, m))
        _dft(L.fdtd_dft_noalloc, xs, dt, fs, -dt / 2)
    assert _free_device_bytes() == before


def test_noalloc_dft_rejects_sizes_beyond_its_limit():
    L = N.lib()
    x = np.zeros(32769)
    f = np.ones(4)
    re, im = np.zeros(4), np.zeros(4)
    rc = L.fdtd_dft_noalloc(N.dptr(x), x.size, 1e-12, N.dptr(f), f.size, 0.0, N.dptr(re), N.dptr(im))
    assert rc == N.FDTD_ERR_BADARG
    assert b"32768" in L.fdtd_last_error()
    f = np.ones(4097)
    re, im = np.zeros(4097), np.zeros(4097)
    rc = L.fdtd_dft_noalloc(N.dptr(x[:10]), 10, 1e-12, N.dptr(f), f.size, 0.0, N.dptr(re), N.dptr(im))
    assert rc == N.FDTD_ERR_BADARG
