"""The any-hit entry point that allocates nothing (pfxt_occluded_noalloc), for
callers whose own allocator owns the device heap or that must not allocate
while GPU work is in flight.  Its blocked flags must equal those of the
device entry point pfxt_occluded_device and the oracle's any-hit walk on two
calls in a row (a larger batch, then a smaller one, so stale scratch from the
first call cannot leak into the second); a call must not lower the device's
free memory; an over-size batch is refused before any GPU work.  This file is
collected last on purpose."""
import numpy as np
import pytest

import oracle
from pfx_b200 import abi, synth
from pfx_b200 import rays as raymix
from pfx_b200.trace import Trace

pytestmark = pytest.mark.gpu


def test_noalloc_occlusion_matches_the_device_entry_point(gpu):
    import torch

    w = synth.small("plain_512", (48, 40))
    trace = Trace(w.scene, w.settings, w.width, w.height)
    ref = oracle.scene_buffers(w.scene, w.settings)
    lib = abi.load()
    stream = torch.cuda.current_stream().cuda_stream
    batches = []
    for seed, n_rays in ((5, 1 << 15), (6, 1 << 12)):
        _, shadow = raymix.pass_mix(trace, w.scene, w.width, w.height, n_rays, seed=seed)
        n = len(shadow)
        d_rays = torch.from_numpy(shadow.view(np.uint8).copy()).cuda()
        d_words = torch.zeros(n, dtype=torch.int32, device="cuda")
        d_bytes = torch.full((n,), 7, dtype=torch.uint8, device="cuda")
        batches.append((shadow, d_rays, d_words, d_bytes))
    torch.cuda.synchronize()
    for k, (shadow, d_rays, d_words, d_bytes) in enumerate(batches):
        n = len(shadow)
        abi.check(lib.pfxt_occluded_device(trace.handle, d_rays.data_ptr(), n, d_words.data_ptr(), stream))
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        abi.check(lib.pfxt_occluded_noalloc(trace.handle, d_rays.data_ptr(), n, d_bytes.data_ptr(), stream))
        torch.cuda.synchronize()
        # driver-level free memory: a cudaMalloc inside the library would show here
        assert torch.cuda.mem_get_info()[0] >= free_before, "the no-allocation call allocated device memory"
        want = d_words.cpu().numpy() != 0
        got = d_bytes.cpu().numpy()
        assert set(np.unique(got).tolist()) <= {0, 1}
        assert np.array_equal(got == 1, want)
        assert np.array_equal(got == 1, oracle.trace(ref, shadow, any_hit=True)["hit"] == 1)
        assert 0.0 < want.mean() < 1.0
    shadow, d_rays, _, d_bytes = batches[0]
    rc = lib.pfxt_occluded_noalloc(trace.handle, d_rays.data_ptr(), abi.NOALLOC_MAX_RAYS + 1, d_bytes.data_ptr(),
                                   stream)
    assert rc == abi.ERR_INVALID
    assert b"at most" in lib.pfxt_last_error()
    trace.close()
