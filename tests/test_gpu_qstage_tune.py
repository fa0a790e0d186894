"""Q-stage commit, LDE plan autotuner and packed-witness commit, through the C-ABI library.

* Q stage: Starks::computeQ (starks.hpp:186-239) run by the reference's own NTT and field code
  (seeded fixtures from the reference CPU build) and restated by the oracle; cmQ words, tree and
  root bit-exact, with q given column-major or row-major.
* Autotuner: every plan computes the same LDE (only speed changes); the table round-trips
  through a file.
* Packed witness: a commit of the bit-packed rows equals the commit of the unpacked trace.
"""
import hashlib
import os
import tempfile

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


@pytest.mark.parametrize("nbits,nbe,qdeg,qdim,arity,rowmajor", [
    (4, 6, 3, 3, 4, True), (6, 7, 2, 3, 4, False), (8, 10, 4, 3, 3, True), (10, 11, 1, 3, 2, True),
    (5, 9, 16, 2, 4, False), (12, 14, 3, 3, 4, True)])
def test_commit_q_matches_oracle(dev, torch_cuda, orc, nbits, nbe, qdeg, qdim, arity, rowmajor):
    torch = torch_cuda
    next_ = 1 << nbe
    q = oracle.random_field((next_, qdim), 40 + nbits + qdeg)
    root_o, cmq_o, tree_o = orc.commit_q(q, nbits, nbe, qdeg, qdim, arity)
    d_q = to_dev(torch, q if rowmajor else q.T.copy())
    ncols = qdeg * qdim
    d_cmq = torch.zeros(next_ * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(dev.tree_num_elements(next_, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(dev.q_scratch_words(nbe, qdim), dtype=torch.int64, device="cuda")
    root = dev.commit_q_device(d_cmq, d_tree, d_q, nbits, nbe, qdeg, qdim, arity, d_scr, q_rowmajor=rowmajor)
    assert (root == root_o).all()
    assert (from_dev(d_cmq).reshape(ncols, next_).T == cmq_o).all()
    assert (from_dev(d_tree) == tree_o).all()


@pytest.mark.parametrize("rowmajor", [True, False])
def test_commit_q_matches_reference_fixtures(dev, torch_cuda, kats, rowmajor):
    """b200_commit_q_device against Starks::computeQ as the reference CPU build computes it
    (tests/golden/reference_kats.json "seeded_q_commits", written by make_golden.py)."""
    torch = torch_cuda
    for c in kats["seeded_q_commits"]:
        nbits, nbe, qdeg, qdim, arity = c["nBits"], c["nBitsExt"], c["qDeg"], c["qDim"], c["arity"]
        next_ = 1 << nbe
        q = oracle.random_field((next_, qdim), c["seed"])
        ncols = qdeg * qdim
        d_q = to_dev(torch, q if rowmajor else q.T.copy())
        d_cmq = torch.zeros(next_ * ncols, dtype=torch.int64, device="cuda")
        d_tree = torch.zeros(dev.tree_num_elements(next_, arity), dtype=torch.int64, device="cuda")
        d_scr = torch.zeros(dev.q_scratch_words(nbe, qdim), dtype=torch.int64, device="cuda")
        root = dev.commit_q_device(d_cmq, d_tree, d_q, nbits, nbe, qdeg, qdim, arity, d_scr, q_rowmajor=rowmajor)
        assert [int(v) for v in root] == c["root"], c
        cmq = np.ascontiguousarray(from_dev(d_cmq).reshape(ncols, next_).T)
        assert hashlib.sha256(cmq.astype("<u8").tobytes()).hexdigest() == c["cmq_sha256"]
        assert hashlib.sha256(from_dev(d_tree).astype("<u8").tobytes()).hexdigest() == c["tree_sha256"]


def test_commit_q_rejects_bad_shapes(dev, torch_cuda):
    torch = torch_cuda
    d = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with pytest.raises(dev.B200Error):  # qDeg above NExt / N
        dev.commit_q_device(d, d, d, 4, 5, 3, 3, 4, d)
    with pytest.raises(dev.B200Error):  # nBitsExt < nBits
        dev.commit_q_device(d, d, d, 6, 5, 1, 3, 4, d)


def test_autotune_keeps_results_and_roundtrips(dev, torch_cuda, orc):
    torch = torch_cuda
    nbits, nbe, ncols, arity = 14, 15, 24, 4
    trace = oracle.random_field((1 << nbits, ncols), 9)
    root_o, _, _ = orc.commit(trace, nbe, arity)
    d_trace = to_dev(torch, trace)
    d_lde = torch.zeros((1 << nbe) * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(dev.tree_num_elements(1 << nbe, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(dev.lde_scratch_words(nbits, ncols), dtype=torch.int64, device="cuda")
    # every plan gives the same root
    for kf, kr in ((8, 8), (12, 12), (9, 11), (12, 7)):
        dev.autotune_set(nbits, nbe, ncols, kf, kr)
        assert dev.autotune_get(nbits, nbe, ncols) == (kf, kr)
        root = dev.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, arity, d_scr)
        assert (root == root_o).all(), (kf, kr)
    ms, kf, kr = dev.autotune_lde(nbits, nbe, ncols)
    assert ms > 0 and 8 <= kf <= 12 and 8 <= kr <= 12
    assert dev.autotune_get(nbits, nbe, ncols) == (kf, kr)
    root = dev.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, arity, d_scr)
    assert (root == root_o).all()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "plans.txt")
        dev.autotune_save(path)
        dev.autotune_set(nbits, nbe, ncols, 8, 8)
        dev.autotune_load(path)
        assert dev.autotune_get(nbits, nbe, ncols) == (kf, kr)


@pytest.mark.parametrize("nbits,nbe,bits,arity", [
    (8, 9, [1, 7, 64, 33, 31, 2, 64, 17, 5], 4), (10, 12, [32] * 20, 3), (6, 7, [64], 2),
    (11, 12, [3, 61, 40, 24, 63, 1, 1, 1, 60, 8, 13], 4),
    (6, 7, [(i * 37) % 64 + 1 for i in range(300)], 4)])  # widths passed as kernel-parameter bytes
def test_packed_commit_equals_plain(dev, torch_cuda, orc, nbits, nbe, bits, arity):
    torch = torch_cuda
    n, ncols = 1 << nbits, len(bits)
    rng = np.random.default_rng(nbits + ncols)
    trace = np.zeros((n, ncols), dtype=np.uint64)
    for c, b in enumerate(bits):
        v = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
        trace[:, c] = v if b == 64 else v & np.uint64((1 << b) - 1)
    packed = dev.pack_rows(trace, bits)
    wpr = dev.packed_words_per_row(bits)
    assert packed.shape == (n, wpr)
    root_o, _, tree_o = orc.commit(trace, nbe, arity)
    d_packed = to_dev(torch, packed)
    d_lde = torch.zeros((1 << nbe) * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(dev.tree_num_elements(1 << nbe, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(dev.lde_scratch_words(nbits, ncols), dtype=torch.int64, device="cuda")
    root = dev.commit_packed_device(d_lde, d_tree, d_packed, wpr, bits, nbits, nbe, arity, d_scr)
    assert (root == root_o).all()
    assert (from_dev(d_tree) == tree_o).all()


def test_packed_commit_rejects_bad_widths(dev, torch_cuda):
    torch = torch_cuda
    d = torch.zeros(1 << 10, dtype=torch.int64, device="cuda")
    with pytest.raises(dev.B200Error):  # a zero-width column
        dev.commit_packed_device(d, d, d, 1, [0, 5], 4, 5, 4, d)
    with pytest.raises(dev.B200Error):  # wider than 64 bits
        dev.commit_packed_device(d, d, d, 2, [65], 4, 5, 4, d)
    with pytest.raises(dev.B200Error):  # words_per_row too small
        dev.commit_packed_device(d, d, d, 1, [40, 40], 4, 5, 4, d)
    with pytest.raises(dev.B200Error):  # more columns than the kernel-parameter table holds
        dev.commit_packed_device(d, d, d, 193, [1] * 12289, 4, 5, 4, d)
