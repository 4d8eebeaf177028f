"""The allocation-free triangle count, gpm_tc_csr_noalloc.

It exists for callers that cannot allocate device memory (a framework that
owns the device through its own pool, services that forbid allocation after
start-up, code that must not trigger an allocation's implicit
synchronisation).  Its scratch is a fixed array inside libgpm.so, so the test
checks it against the allocating entry point on the same device-resident
graph, twice in a row (the second call must not see the first call's queue
state), and checks that oversized graphs are refused before any launch.

The file is named to run last: a failure here leaves every other test
already run, and the test also passes alone in a fresh process (its first
call performs the per-device set-up).
"""
import ctypes

import numpy as np
import pytest

import gpm

pytestmark = pytest.mark.gpu


def _call(n, off_t, idx_t, out_t, stream):
    return gpm.lib.gpm_tc_csr_noalloc(n, ctypes.c_void_p(off_t.data_ptr()), ctypes.c_void_p(idx_t.data_ptr()),
                                      ctypes.c_void_p(stream), ctypes.c_void_p(out_t.data_ptr()))


@pytest.mark.parametrize("scale,relabel", [(16, False), (18, True)])
def test_noalloc_matches_allocating_entry_point(scale, relabel):
    import torch
    g = gpm.Graph.rmat(scale, 16, seed=scale).orient(relabel=relabel)
    off, idx = g.csr()
    dev = torch.device("cuda", 0)
    off_t = torch.from_numpy(off).to(dev)
    idx_t = torch.from_numpy(idx).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ref = torch.zeros(1, dtype=torch.int64, device=dev)
    g.tc_async(gpm.TC_HASH, stream, ref.data_ptr())
    torch.cuda.synchronize()
    want = int(ref.item())
    assert want == g.tc(gpm.V_CENTRIC) > 0
    outs = [torch.full((1,), -1, dtype=torch.int64, device=dev) for _ in range(3)]
    gpm.check(_call(len(off) - 1, off_t, idx_t, outs[0], stream))  # first call: per-device set-up
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for out in outs[1:]:
        gpm.check(_call(len(off) - 1, off_t, idx_t, out, stream))
        torch.cuda.synchronize()
    # device memory in use is unchanged by the later calls: they allocated nothing
    assert torch.cuda.mem_get_info(dev)[0] == free_before
    assert [int(o.item()) for o in outs] == [want] * 3


def test_noalloc_rejects_oversized_graph():
    import torch
    dev = torch.device("cuda", 0)
    off_t = torch.zeros(2, dtype=torch.int64, device=dev)
    idx_t = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.zeros(1, dtype=torch.int64, device=dev)
    status = _call((1 << 20) + 1, off_t, idx_t, out, torch.cuda.current_stream(dev).cuda_stream)
    assert status == 1  # GPM_EINVAL
    assert b"1048576" in gpm.lib.gpm_last_error()
