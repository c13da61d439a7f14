"""flip_inclusive_scan_u32_noalloc: the inclusive scan for callers that cannot
allocate device memory (a host that owns a fixed device-memory budget, or a
per-frame callback that must not pay cudaMalloc's implicit synchronisation).
It keeps its scratch in a static device array of the library instead of
taking caller scratch.  Checked through the C ABI against the allocating
entry point, flip_inclusive_scan_u32, on two calls in a row: the second call
must not see the first call's leftover look-back words.  This file is
collected last so that a run stopping at its first failure has already run
every other test."""
import ctypes as C

import numpy as np
import pytest

import flip2_b200 as F

pytestmark = pytest.mark.gpu


def _scan_both(torch, x):
    L = F.lib()
    d_in = torch.from_numpy(x.view(np.int32)).cuda()
    ref = torch.empty_like(d_in)
    out = torch.empty_like(d_in)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    nb = L.flip_inclusive_scan_scratch_bytes(x.size)
    scratch = torch.empty(nb, dtype=torch.uint8, device="cuda")
    assert L.flip_inclusive_scan_u32(C.c_void_p(d_in.data_ptr()), C.c_void_p(ref.data_ptr()), x.size,
                                     C.c_void_p(scratch.data_ptr()), nb, stream) == 0
    assert L.flip_inclusive_scan_u32_noalloc(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), x.size,
                                             stream) == 0
    torch.cuda.synchronize()
    return ref.cpu().numpy().view(np.uint32), out.cpu().numpy().view(np.uint32)


def test_noalloc_scan_matches_allocating_scan_twice():
    import torch
    assert torch.cuda.is_available()
    rng = np.random.default_rng(11)
    # first call larger than the second, so stale look-back words of the first
    # call would corrupt the second if they were not cleared
    for n in (3_000_001, 1_048_577):
        x = rng.integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
        ref, out = _scan_both(torch, x)
        assert np.array_equal(out, ref)  # bit-exact, like every u32 scan test
        assert np.array_equal(out, np.cumsum(x.astype(np.uint64)).astype(np.uint32))


def test_noalloc_scan_rejects_sizes_beyond_its_static_scratch():
    L = F.lib()
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    assert L.flip_inclusive_scan_u32_noalloc(dummy, dummy, (1 << 28) + 1, None) == 1
    assert b"2^28" in L.flip_last_error(None)


def test_noalloc_scan_status_reports_no_timeout_after_good_calls():
    import torch
    L = F.lib()
    x = np.arange(50_000, dtype=np.uint32)
    _scan_both(torch, x)
    flags = C.c_uint32(0xFFFFFFFF)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.flip_inclusive_scan_u32_noalloc_status(stream, C.byref(flags)) == 0
    assert flags.value == 0


@pytest.mark.parametrize("n", [(1 << 28) - 4096, (1 << 28) - 4095, 1 << 28])
def test_noalloc_scan_at_its_size_limit(n):
    """2^28 elements fill every status word of the static array (65,536 tiles
    of 4096); 2^28 - 4095 reaches the last word with a one-element tile, and
    2^28 - 4096 stops one tile short of it.  All-ones input: the scan is
    1, 2, ..., n."""
    import torch
    L = F.lib()
    d_in = torch.ones(n, dtype=torch.int32, device="cuda")
    out = torch.empty_like(d_in)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.flip_inclusive_scan_u32_noalloc(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), n, stream) == 0
    flags = C.c_uint32(0)
    assert L.flip_inclusive_scan_u32_noalloc_status(stream, C.byref(flags)) == 0 and flags.value == 0
    expect = torch.arange(1, n + 1, dtype=torch.int32, device="cuda")
    assert torch.equal(out, expect)
    del d_in, out, expect
    torch.cuda.empty_cache()
