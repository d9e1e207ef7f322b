"""Host-to-device copies by the SMs (dwba_copy_from_host) and the staging ring that uploads a call's
descriptor arrays through them.

The copy must reproduce the bytes exactly for any size and alignment and refuse memory of the wrong
kind (pageable host memory, device memory as the source), and the ring must keep every array intact
when it wraps around while earlier copies are still queued.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _lib():
    from dwba_b200 import _lib
    return _lib, _lib.load()


def test_copy_from_pinned_host_memory_is_exact():
    L, lib = _lib()
    rng = np.random.default_rng(3)
    src = torch.empty(1 << 20, dtype=torch.uint8, pin_memory=True)
    src.numpy()[:] = rng.integers(0, 256, size=1 << 20, dtype=np.uint8)
    dst = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for off, n in ((0, 1 << 20), (16, 4096), (3, 1001), (0, 1), (64, 48)):
        dst.zero_()
        rc = lib.dwba_copy_from_host(dst.data_ptr() + off, src.data_ptr() + off, n, st)
        assert rc == L.DWBA_OK
        torch.cuda.synchronize()
        got = dst.cpu().numpy()
        assert np.array_equal(got[off:off + n], src.numpy()[off:off + n])
        assert not got[:off].any() and not got[off + n:].any()


def test_copy_refuses_memory_the_device_cannot_address():
    L, lib = _lib()
    st = torch.cuda.current_stream().cuda_stream
    dst = torch.zeros(4096, dtype=torch.uint8, device="cuda")
    pageable = np.ones(4096, dtype=np.uint8)
    assert lib.dwba_copy_from_host(dst.data_ptr(), pageable.ctypes.data, 4096, st) == L.DWBA_ERR_INVALID_ARG
    # a source that is device memory, not host memory; null pointers and a negative size
    assert lib.dwba_copy_from_host(dst.data_ptr(), dst.data_ptr(), 16, st) == L.DWBA_ERR_INVALID_ARG
    pinned = torch.ones(4096, dtype=torch.uint8, pin_memory=True)
    assert lib.dwba_copy_from_host(None, pinned.data_ptr(), 16, st) == L.DWBA_ERR_INVALID_ARG
    assert lib.dwba_copy_from_host(dst.data_ptr(), None, 16, st) == L.DWBA_ERR_INVALID_ARG
    assert lib.dwba_copy_from_host(dst.data_ptr(), pinned.data_ptr(), -1, st) == L.DWBA_ERR_INVALID_ARG
    torch.cuda.synchronize()
    assert not dst.cpu().numpy().any()


def test_staging_ring_keeps_arrays_intact_across_wraps():
    from dwba_b200.engine import _dev, _Staging
    rng = np.random.default_rng(5)
    xs = [rng.standard_normal(int(n)) for n in rng.integers(1, (3 << 20) // 8, size=90)]
    xs += [rng.integers(-5, 5, size=7, dtype=np.int64), np.arange(12, dtype=np.int32).reshape(3, 4)]
    assert sum(x.nbytes for x in xs) > 2 * _Staging.SIZE  # the ring wraps at least twice
    outs = [_dev(x, torch.device("cuda")) for x in xs]
    for x, o in zip(xs, outs):
        assert o.dtype == torch.from_numpy(x).dtype and tuple(o.shape) == x.shape
        assert np.array_equal(o.cpu().numpy(), x)
