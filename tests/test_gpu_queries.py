"""FRI query openings read from the resident LDE and tree, against the oracle.

An opening is MerkleTreeGL::getGroupProof (merkleTreeGL.cpp:145-175): row values, then the
sibling digests level by level (to the root, or to a level of <= arity^llv nodes).  Checked word
for word against the oracle's restatement, and by hashing every opening back to the root.
Calls go through the C-ABI library; torch only allocates device memory.
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


@pytest.fixture(scope="module")
def dev(pkg, torch_cuda):
    pkg.init(0)
    return pkg


def to_dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint64).view(np.int64)).cuda()


def from_dev(t):
    return t.cpu().numpy().view(np.uint64)


def _commit(dev, torch, nbits, nbe, ncols, arity, seed):
    trace = oracle.random_field((1 << nbits, ncols), seed)
    d_trace = to_dev(torch, trace)
    d_lde = torch.zeros((1 << nbe) * max(ncols, 1), dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(dev.tree_num_elements(1 << nbe, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(max(dev.lde_scratch_words(nbits, ncols), 1), dtype=torch.int64, device="cuda")
    root = dev.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, arity, d_scr)
    return trace, d_lde, d_tree, root


@pytest.mark.parametrize("nbits,nbe,ncols,arity,llv", [
    (8, 9, 13, 4, 0), (8, 10, 5, 3, 0), (7, 8, 12, 2, 0), (10, 11, 40, 4, 2), (9, 10, 3, 2, 3), (6, 7, 1, 4, 1)])
def test_openings_match_oracle(dev, torch_cuda, orc, nbits, nbe, ncols, arity, llv):
    torch = torch_cuda
    trace, d_lde, d_tree, root = _commit(dev, torch, nbits, nbe, ncols, arity, 11 + nbits + ncols)
    next_ = 1 << nbe
    lde = from_dev(d_lde)[: next_ * ncols].reshape(ncols, next_).T.copy()  # row-major copy
    tree = from_dev(d_tree)
    rng = np.random.default_rng(5)
    rows = np.concatenate([[0, next_ - 1], rng.integers(0, next_, 30)]).astype(np.uint64)
    words = dev.query_proof_words(next_, ncols, arity, llv)
    d_rows = to_dev(torch, rows)
    d_out = torch.zeros(len(rows) * words, dtype=torch.int64, device="cuda")
    dev.query_openings_device(d_out, d_lde, next_, ncols, d_tree, arity, d_rows, len(rows), llv=llv)
    torch.cuda.synchronize()
    out = from_dev(d_out).reshape(len(rows), words)
    for i, r in enumerate(rows):
        exp = orc.group_proof(lde, tree, arity, int(r), llv)
        assert len(exp) == words
        assert (out[i] == exp).all(), (i, int(r))
        if llv == 0:
            assert (orc.root_from_proof(out[i], ncols, next_, arity, int(r)) == root).all()


def test_openings_zero_queries_and_bad_arity(dev, torch_cuda):
    torch = torch_cuda
    trace, d_lde, d_tree, root = _commit(dev, torch, 6, 7, 4, 4, 3)
    d_out = torch.zeros(8, dtype=torch.int64, device="cuda")
    d_rows = torch.zeros(1, dtype=torch.int64, device="cuda")
    dev.query_openings_device(d_out, d_lde, 128, 4, d_tree, 4, d_rows, 0)
    with pytest.raises(dev.B200Error):
        dev.query_openings_device(d_out, d_lde, 128, 4, d_tree, 5, d_rows, 1)
    assert dev.query_proof_words(128, 4, 4, 0) == 4 + 4 * 3 * 4  # 128 -> 32 -> 8 -> 2 -> 1: 4 levels
