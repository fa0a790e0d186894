"""Cooperative Poseidon2 / Poseidon1 kernels (coop.cuh) at the boundaries where the tree builder
switches between them and the one-thread-per-state kernels.

merkle::build_tree hashes the leaves cooperatively up to 8192 rows, builds levels of up to 8192
parents cooperatively, and runs the last levels (<= 64 parents at W12/W16, <= 128 at W8) in one
single-CTA launch.  Every case compares the whole tree buffer (leaves, padding, every level) with
the oracle's restatement of Poseidon2GoldilocksGPU::merkletree (poseidon2_goldilocks.cpp:129-175)
or, for hash family 1, of PoseidonGoldilocks::merkletree (poseidon_goldilocks.cpp).
Calls go through the C-ABI library; torch only allocates device memory.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.init(0)
    return pkg, torch


def _tree(dev, m, arity):
    pkg, torch = dev
    nrows, ncols = m.shape
    src = m.T.copy() if ncols else np.zeros(1, np.uint64)
    d_src = torch.from_numpy(np.ascontiguousarray(src).view(np.int64)).cuda()
    d_tree = torch.zeros(pkg.tree_num_elements(nrows, arity), dtype=torch.int64, device="cuda")
    pkg.merkletree_device(d_tree, d_src, 1, nrows, ncols, nrows, arity)
    torch.cuda.synchronize()
    return d_tree.cpu().numpy().view(np.uint64)


# (nrows, ncols, arity): leaf switch at 8192 rows; level switch at 8192 parents; tail limits
# 64 parents (arity 3, 4) and 128 parents (arity 2); sponges of 1, 2 and 3 permutations
CASES = [
    (8192, 13, 4), (8193, 13, 4),          # cooperative / one-thread leaves, then cooperative levels
    (32768, 3, 4), (32772, 3, 4),          # 8192 parents (cooperative) / 8193 (one-thread level)
    (256, 25, 4), (257, 25, 4),            # straight into the tail / one cooperative level first
    (192, 9, 3), (193, 9, 3), (8193, 8, 3),
    (256, 5, 2), (257, 5, 2), (16386, 4, 2),
    (1, 7, 4), (2, 0, 4), (5, 30, 2),
]


@pytest.mark.parametrize("nrows,ncols,arity", CASES)
def test_tree_matches_oracle_at_switch_points(dev, orc, nrows, ncols, arity):
    m = oracle.random_field((nrows, ncols), nrows * 7 + ncols + arity)
    if nrows > 4:
        m[:3] = np.uint64(oracle.P - 1)  # loose-arithmetic edge values in the first rows
    got = _tree(dev, m, arity)
    exp = orc.merkletree(m, arity)
    assert got.shape == exp.shape
    bad = np.nonzero(got != exp)[0]
    assert bad.size == 0, (nrows, ncols, arity, bad[:8])


@pytest.fixture(scope="module")
def orc1():
    return oracle.Oracle(family=1)


# Poseidon1: the same switch points (the oracle's Poseidon1 trees are slower, so fewer large ones)
CASES1 = [(8192, 13, 4), (8193, 13, 4), (256, 25, 4), (257, 25, 4), (192, 9, 3), (193, 9, 3),
          (256, 5, 2), (257, 5, 2), (1, 7, 4), (2, 0, 4), (5, 30, 2), (32772, 3, 4)]


@pytest.mark.parametrize("nrows,ncols,arity", CASES1)
def test_poseidon1_tree_matches_oracle_at_switch_points(dev, orc1, nrows, ncols, arity):
    pkg, _ = dev
    m = oracle.random_field((nrows, ncols), nrows * 11 + ncols + arity)
    if nrows > 4:
        m[:3] = np.uint64(oracle.P - 1)
    pkg.set_native_hash_family(1)
    try:
        got = _tree(dev, m, arity)
    finally:
        pkg.set_native_hash_family(2)
    exp = orc1.merkletree(m, arity)
    bad = np.nonzero(got != exp)[0]
    assert bad.size == 0, (nrows, ncols, arity, bad[:8])
