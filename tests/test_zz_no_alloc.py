"""The allocation-free LDE entry point (b200_lde_device_static_scratch).

It serves callers that may not allocate device memory: a prover whose device memory all
comes from its own pool or budget, or a latency-critical loop that cannot pay cudaMalloc's
implicit synchronisation.  Its scratch is a fixed 64 MiB array inside the library, shared
by every call.  Two calls in a row, with different shapes (so the second sees the first
call's leftovers in the shared array), must give exactly what the allocating entry point
b200_lde_device gives; shapes above the built-in size are rejected.  Bit-exact comparison
(integer field arithmetic, no tolerance).

This file sorts last so that a run stopping at its first failure has run every other test.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint64).view(np.int64)).cuda()


def test_static_scratch_lde_matches_allocating_entry_point(pkg, torch_cuda):
    torch = torch_cuda
    pkg.init(0)
    cases = [(14, 15, 40, True, 11), (16, 18, 100, False, 12)]  # N * nCols: 655360, 6553600 <= 2^23
    for nb, nbe, nc, rowmajor, seed in cases:
        trace = oracle.random_field((1 << nb, nc), seed)
        d_trace = _dev(torch, trace if rowmajor else trace.T.copy())
        d_ref = torch.zeros((nc << nbe,), dtype=torch.int64, device="cuda")
        d_new = torch.full((nc << nbe,), -1, dtype=torch.int64, device="cuda")
        d_scr = torch.zeros((pkg.lde_scratch_words(nb, nc),), dtype=torch.int64, device="cuda")
        pkg.lde_device(d_ref, d_trace, nb, nbe, nc, d_scr, trace_rowmajor=rowmajor)
        pkg.lde_device_static_scratch(d_new, d_trace, nb, nbe, nc, trace_rowmajor=rowmajor)
        torch.cuda.synchronize()
        assert torch.equal(d_ref, d_new), (nb, nbe, nc)


def test_static_scratch_rejects_oversize(pkg, torch_cuda):
    pkg.init(0)
    d = torch_cuda.zeros((8,), dtype=torch_cuda.int64, device="cuda")
    with pytest.raises(pkg.B200Error) as e:
        pkg.lde_device_static_scratch(d, d, 22, 23, 3)  # 3 * 2^22 words > 2^23
    assert e.value.code == pkg.B200_EINVAL
    assert "2^23" in str(e.value)
