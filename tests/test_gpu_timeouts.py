"""The bounded device waits give up and report, and the GPU stays usable.

The sort's and the scan's decoupled look-back poll their predecessor tile's
status word a bounded number of times.  flip_test_lookback_timeout runs each
with tile 0 never claimed, so tile 1 polls a word that nothing publishes: the
wait must run out after the given number of polls, the kernel must return,
the scratch's error word must carry the timeout bit, flip_scratch_status must
return FLIP_ERR_TIMEOUT -- and afterwards the same kernels must still give
exact results in the same context.  Nothing here faults or hangs the GPU: the
waits end by construction and every access stays inside the buffers."""
import ctypes as C

import numpy as np
import pytest

import flip2_b200 as F

pytestmark = pytest.mark.gpu
FLIP_ERR_TIMEOUT = 4


@pytest.mark.parametrize("which", [0, 1])
def test_lookback_wait_times_out_and_reports(which):
    import torch
    L = F.lib()
    n = 5 * 4096 + 17
    keys = np.random.default_rng(3).integers(0, 2 ** 32, size=n, dtype=np.uint64).astype(np.uint32)
    d_in = torch.from_numpy(keys.view(np.int32)).cuda()
    ok = torch.empty_like(d_in)
    ov = torch.empty_like(d_in)
    nb = max(L.flip_sort_pairs_scratch_bytes(n), L.flip_inclusive_scan_scratch_bytes(n))
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    flags = C.c_uint32(0)
    rc = L.flip_test_lookback_timeout(which, C.c_void_p(d_in.data_ptr()), C.c_void_p(ok.data_ptr()),
                                      C.c_void_p(ov.data_ptr()), n, 2000, C.c_void_p(scr.data_ptr()), nb, stream,
                                      C.byref(flags))
    assert rc == FLIP_ERR_TIMEOUT, rc
    assert flags.value & 1
    assert b"timed out" in L.flip_last_error(None)
    torch.cuda.synchronize()  # the kernels returned: the context is still usable
    # the same kernels, unhooked, in the same context: exact again, status clean
    if which == 0:
        out, s = F.inclusive_scan(d_in, return_scratch=True)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), np.cumsum(keys.astype(np.uint64)).astype(np.uint32))
    else:
        k2, v2, s = F.sort_pairs(d_in, key_bits=32, return_scratch=True)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k2.cpu().numpy().view(np.uint32), keys[order])
        assert np.array_equal(v2.cpu().numpy().view(np.uint32), order.astype(np.uint32))
    flags = C.c_uint32(0xFFFF)
    assert L.flip_scratch_status(C.c_void_p(s.data_ptr()), stream, C.byref(flags)) == 0
    assert flags.value == 0


def test_engine_step_reports_clean_error_word():
    """A native step leaves the engine's device error word clear, and the
    synchronising calls that check it return FLIP_OK."""
    from flip2_b200 import scenes
    pos, vel = scenes.dam_break(16, seed=0)
    P = F.Particles(pos.shape[0], mode=F.MODE_NATIVE)
    P.setDomain(0.0, 0.0, 0.0, 4, 4, 4, 0.25)
    P.upload(pos, vel)
    P.step(1.0 / 240)
    P.sync()
    assert P.info().error_flags == 0
    P.close()
