"""The allocation-free LDE entry point (b200_lde_device_static_scratch).

It serves callers that may not allocate device memory: a prover whose device memory all
comes from its own pool or budget, or a latency-critical loop that cannot pay cudaMalloc's
implicit synchronisation.  Its scratch is a fixed 64 MiB array inside the library, shared
by every call.  Calls in a row with different shapes — the largest first, so the later ones run
over its leftovers in the shared array, one of them on a stream of the caller's, one exactly at the
2^23-word limit — must give exactly what the allocating entry point b200_lde_device gives; a shape
one column past the limit is rejected.  Bit-exact comparison (integer field arithmetic, no
tolerance).

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
    side = torch.cuda.Stream()
    # (nBits, nBitsExt, nCols, row-major input, seed, caller stream): N * nCols = 2^23 (the limit),
    # 6553600 and 655360 words
    cases = [(17, 18, 64, True, 13, None), (16, 18, 100, False, 12, side), (14, 15, 40, True, 11, None)]
    for nb, nbe, nc, rowmajor, seed, stream in cases:
        trace = oracle.random_field((1 << nb, nc), seed)
        d_trace = _dev(torch, trace if rowmajor else trace.T.copy())
        d_ref = torch.zeros((nc << nbe,), dtype=torch.int64, device="cuda")
        d_new = torch.full((nc << nbe,), -1, dtype=torch.int64, device="cuda")
        d_scr = torch.zeros((pkg.lde_scratch_words(nb, nc),), dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        pkg.lde_device(d_ref, d_trace, nb, nbe, nc, d_scr, trace_rowmajor=rowmajor)
        pkg.lde_device_static_scratch(d_new, d_trace, nb, nbe, nc, trace_rowmajor=rowmajor,
                                      stream=None if stream is None else stream.cuda_stream)
        if stream is not None:
            stream.synchronize()
        torch.cuda.synchronize()
        assert torch.equal(d_ref, d_new), (nb, nbe, nc)


def test_static_scratch_rejects_oversize(pkg, torch_cuda):
    pkg.init(0)
    d = torch_cuda.zeros((8,), dtype=torch_cuda.int64, device="cuda")
    for nb, nbe, nc in ((22, 23, 3), (17, 18, 65)):  # 3 * 2^22 and 2^23 + 2^17 words > 2^23
        with pytest.raises(pkg.B200Error) as e:
            pkg.lde_device_static_scratch(d, d, nb, nbe, nc)
        assert e.value.code == pkg.B200_EINVAL
        assert "2^23" in str(e.value)
