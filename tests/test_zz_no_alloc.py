"""mgm_avg_dx_noalloc: the average-spacing entry point for callers that cannot
let the library allocate device memory (memory owned by another allocator or
a fixed arena).  It must give exactly what mgm_avg_dx gives, call after call,
using only the caller's device buffers and the library's fixed scratch array.

This file is collected last on purpose: a failure here leaves every other
test already run."""
import numpy as np
import pytest

from multigrid_meshless_b200 import _lib, api, clouds


def test_noalloc_rejects_oversize_before_touching_the_gpu():
    L = _lib.load()
    st = L.mgm_avg_dx_noalloc(_lib.NOALLOC_MAX_NODES + 1, 20, 2, None, None, None, None, None, None, None)
    assert st == _lib.MGM_ERR_ARG
    assert b"exceeds the fixed scratch" in L.mgm_last_error()


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_two_calls(require_gpu):
    """Two calls in a row, the second on a non-default stream: each gives the
    bits of mgm_avg_dx, and the second (the scratch array is resident after
    the first) leaves the device's free memory unchanged."""
    import torch

    L = _lib.load()
    side = torch.cuda.Stream()
    for call, (m, k, seed) in enumerate(((120, 20, 3), (90, 30, 4))):
        c = clouds.cavity2d(m, seed=seed)
        cloud = api.knn_cloud(c.x, c.y, c.z, c.btag, c.nb, k, 2)
        want = api.avg_dx(c.x, c.y, c.z, c.btag, cloud, 2)
        dev = {nm: torch.from_numpy(np.ascontiguousarray(getattr(c, nm))).cuda() for nm in ("x", "y", "z")}
        bt = torch.from_numpy(np.ascontiguousarray(c.btag, dtype=np.uint8)).cuda()
        cl = torch.from_numpy(np.ascontiguousarray(cloud, dtype=np.int32)).cuda()
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        stream = None if call == 0 else side.cuda_stream
        free_before = torch.cuda.mem_get_info()[0]
        st = L.mgm_avg_dx_noalloc(c.n, k, 2, dev["x"].data_ptr(), dev["y"].data_ptr(), dev["z"].data_ptr(),
                                  bt.data_ptr(), cl.data_ptr(), out.data_ptr(), stream)
        assert st == _lib.MGM_OK, L.mgm_last_error()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        if call > 0:
            assert free_after == free_before, (free_before, free_after)
        assert out.item() == want, (call, out.item(), want)
