"""The TMA-staged transpose in front of the LDE (transpose_tma_kernel; the reference's
fromRowMajorToColMajor, goldilocks_tooling.cu:28-59).

Row-major traces of even column counts take the TMA path (two 32 x 16 bulk tensor copies per tile,
128-byte swizzle, bounded barrier wait); odd column counts and unaligned sources take the
thread-loaded tiles.  Both must give the oracle's LDE word for word, edge tiles included (rows and
columns that are not multiples of 32), and no tile copy may miss its wait bound.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.init(0)
    return torch


def _dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint64).view(np.int64)).cuda()


@pytest.mark.parametrize("nb,nbe,nc", [(3, 4, 2), (4, 5, 6), (5, 6, 34), (10, 11, 48), (12, 13, 66), (16, 17, 64),
                                       (12, 14, 31), (13, 14, 2)])
def test_tma_transpose_lde_matches_oracle(pkg, torch_cuda, orc, nb, nbe, nc):
    torch = torch_cuda
    lib = pkg.load()
    trace = oracle.random_field((1 << nb, nc), 300 + nb + nc)
    want = orc.lde(trace, nbe)
    d_trace = _dev(torch, trace)
    outs = []
    prev = lib.b200_set_transpose_tma(1)
    try:
        for tma in (1, 0):
            lib.b200_set_transpose_tma(tma)
            d_lde = torch.full((nc << nbe,), -1, dtype=torch.int64, device="cuda")
            d_scr = torch.zeros((pkg.lde_scratch_words(nb, nc),), dtype=torch.int64, device="cuda")
            pkg.lde_device(d_lde, d_trace, nb, nbe, nc, d_scr)
            torch.cuda.synchronize()
            outs.append(d_lde.cpu().numpy().view(np.uint64).reshape(nc, 1 << nbe).T)
    finally:
        lib.b200_set_transpose_tma(prev)
    assert lib.b200_tma_wait_errors() == 0
    assert (outs[0] == want).all()
    assert (outs[1] == want).all()


def test_tma_transpose_unaligned_source_falls_back(pkg, torch_cuda, orc):
    """A source one word past a 16-byte boundary cannot be a TMA tensor: the thread-loaded tiles run."""
    torch = torch_cuda
    nb, nbe, nc = 8, 9, 10
    trace = oracle.random_field((1 << nb, nc), 77)
    buf = torch.zeros(((1 << nb) * nc + 1,), dtype=torch.int64, device="cuda")
    buf[1:] = _dev(torch, trace.reshape(-1))
    d_lde = torch.zeros((nc << nbe,), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros((pkg.lde_scratch_words(nb, nc),), dtype=torch.int64, device="cuda")
    pkg.lde_device(d_lde, buf.data_ptr() + 8, nb, nbe, nc, d_scr)
    torch.cuda.synchronize()
    assert (d_lde.cpu().numpy().view(np.uint64).reshape(nc, 1 << nbe).T == orc.lde(trace, nbe)).all()
