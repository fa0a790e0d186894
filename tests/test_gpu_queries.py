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


def _verify_to_level(orc, opening, ncols, nrows, arity, row, level, llv):
    """verifyGroupProof with last_level_verification (merkleTreeGL.cpp:177-216): the row's linear
    hash combined with the siblings up to the kept level, compared with that level's node."""
    w = 4 * arity
    h = orc.linear_hash(w, opening[:ncols])
    sib = opening[ncols:]
    idx, n, stop = row, nrows, arity ** llv
    while n > stop:
        cur = idx % arity
        st = np.zeros(w, dtype=np.uint64)
        p = 0
        for i in range(arity):
            if i == cur:
                st[4 * i:4 * i + 4] = h
            else:
                st[4 * i:4 * i + 4] = sib[4 * p:4 * p + 4]
                p += 1
        sib = sib[4 * (arity - 1):]
        h = orc.permute(st)[:4]
        idx //= arity
        n = (n + arity - 1) // arity
    return (h == level[4 * idx:4 * idx + 4]).all()


@pytest.mark.parametrize("nbits,nbe,ncols,arity", [(8, 9, 7, 4), (9, 10, 3, 2), (8, 10, 12, 3)])
def test_last_level_and_openings_verify(dev, torch_cuda, orc, nbits, nbe, ncols, arity):
    torch = torch_cuda
    trace, d_lde, d_tree, root = _commit(dev, torch, nbits, nbe, ncols, arity, 70 + nbits)
    next_ = 1 << nbe
    lde = from_dev(d_lde)[: next_ * ncols].reshape(ncols, next_).T.copy()
    tree = from_dev(d_tree)
    for llv in (1, 2, 3):
        words = dev.load().b200_tree_last_level_words(arity, llv)
        d_level = torch.full((words,), -1, dtype=torch.int64, device="cuda")
        dev.tree_last_level_device(d_level, d_tree, next_, arity, llv)
        torch.cuda.synchronize()
        level = from_dev(d_level)
        # restatement of getLevel over the host copy of the tree
        n, off = next_, 0
        while n > arity ** llv:
            n = (n + arity - 1) // arity
            off += n * arity * 4
        exp = np.zeros(words, dtype=np.uint64)
        exp[:4 * n] = tree[off:off + 4 * n]
        assert (level == exp).all(), llv
        for row in (0, 3, next_ - 1):
            opening = orc.group_proof(lde, tree, arity, row, llv)
            assert _verify_to_level(orc, opening, ncols, next_, arity, row, level, llv), (llv, row)


@pytest.mark.parametrize("n,arity", [(1, 4), (5, 2), (12, 3), (100, 4), (4097, 2)])
def test_merkletree_reduce_device(dev, torch_cuda, orc, refcpu, n, arity):
    torch = torch_cuda
    digests = oracle.random_field((4 * n,), n + arity)
    d_tree = torch.zeros(dev.tree_num_elements(n, arity), dtype=torch.int64, device="cuda")
    root = dev.merkletree_reduce_device(to_dev(torch, digests), n, arity, d_tree)
    assert (root == orc.merkletree_reduce(4 * arity, digests, arity)).all()
    assert (root == refcpu.merkletree_reduce(4 * arity, digests, arity)).all()


def test_merkletree_reduce_golden(dev, torch_cuda, kats):
    torch = torch_cuda
    digests = np.arange(1, 13, dtype=np.uint64)
    d_tree = torch.zeros(dev.tree_num_elements(3, 3), dtype=torch.int64, device="cuda")
    root = dev.merkletree_reduce_device(to_dev(torch, digests), 3, 3, d_tree)
    assert [int(v) for v in root] == kats["poseidon2"]["MERKLETREE_REDUCE_W12_AR3_GOLDEN"]
