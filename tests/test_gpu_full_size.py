"""Parity at the workloads' full row counts (C2: 2^22 -> 2^23 rows at blowup 2; C4: 2^20 -> 2^22
at blowup 4), where the NTT runs its largest windows and the tree its deepest levels.

* Bit-exact against the oracle (NTT_Goldilocks::LDE, ntt_goldilocks.cpp:369-404, and the
  Poseidon2 row sponge and arity-4 tree, poseidon2_goldilocks.cpp:42-175) for a few columns:
  root, every LDE word and every tree node.
* A size-independent property for many columns: the LDE is linear, LDE(x + y) = LDE(x) + LDE(y)
  (mod p), checked word for word.
* At the full C4 and C2 shapes (all columns): the reference-facing commit_witness path and the
  one-pass device path give the same root.
Calls go through the C-ABI library; torch only allocates device memory.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

P = np.uint64(oracle.P)


@pytest.fixture(scope="module")
def dev(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.init(0)
    pkg.set_native_hash_family(2)
    return pkg, torch


def _commit(dev, trace, nbits, nbe, arity=4):
    pkg, torch = dev
    n, ncols = trace.shape
    d_trace = torch.from_numpy(np.ascontiguousarray(trace).view(np.int64)).cuda()
    d_lde = torch.empty((1 << nbe) * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.empty(pkg.tree_num_elements(1 << nbe, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.empty(pkg.lde_scratch_words(nbits, ncols), dtype=torch.int64, device="cuda")
    root = pkg.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, arity, d_scr)
    torch.cuda.synchronize()
    lde = d_lde.cpu().numpy().view(np.uint64).reshape(ncols, 1 << nbe)  # column-major
    tree = d_tree.cpu().numpy().view(np.uint64)
    return root, lde, tree


@pytest.mark.parametrize("nbits,nbe,ncols", [(22, 23, 4), (20, 22, 3)])
def test_full_row_count_matches_oracle(dev, orc, nbits, nbe, ncols):
    trace = oracle.random_field((1 << nbits, ncols), 2200 + nbe)
    root, lde, tree = _commit(dev, trace, nbits, nbe)
    r_o, lde_o, tree_o = orc.commit(trace, nbe, 4)
    assert (root == r_o).all()
    assert (lde.T == lde_o).all()
    assert (tree == tree_o).all()


def _addmod(a, b):
    """(a + b) mod p for canonical uint64 arrays"""
    s = a + b  # wraps when a + b >= 2^64
    wrapped = s < a
    s = np.where(wrapped, s + np.uint64(0xFFFFFFFF), s)  # 2^64 = 2^32 - 1 (mod p); cannot wrap again
    return np.where(s >= P, s - P, s)


def test_full_size_lde_is_linear(dev):
    nbits, nbe, ncols = 22, 23, 32
    x = oracle.random_field((1 << nbits, ncols), 31)
    y = oracle.random_field((1 << nbits, ncols), 32)
    z = _addmod(x, y)
    _, lx, _ = _commit(dev, x, nbits, nbe)
    _, ly, _ = _commit(dev, y, nbits, nbe)
    _, lz, _ = _commit(dev, z, nbits, nbe)
    assert (lz == _addmod(lx, ly)).all()


@pytest.mark.parametrize("nbits,nbe,ncols", [(20, 22, 780), (22, 23, 256)])
def test_full_size_commit_witness_equals_one_pass(dev, nbits, nbe, ncols):
    """At the full C4 (2^20 x 780, blowup 4) and C2 (2^22 x 256, blowup 2) shapes, commit_witness
    from pinned host memory (column blocks of 16, 24, 48, then 64, crossing PCIe while earlier
    blocks are extended; the sponge absorbed in 12-column chunks on the idle device) gives the root
    of the one-pass device commit (transpose, LDE, one leaf kernel).  Both are pinned to the oracle at
    smaller sizes; here they must agree with each other on every bit of the root."""
    import ctypes
    pkg, torch = dev
    N, NExt = 1 << nbits, 1 << nbe
    d_trace = torch.empty(N * ncols, dtype=torch.int64, device="cuda")
    pkg.fill_random_device(d_trace, N * ncols, 780 + nbits)
    d_lde = torch.empty(NExt * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.empty(pkg.tree_num_elements(NExt, 4), dtype=torch.int64, device="cuda")
    d_scr = torch.empty(pkg.lde_scratch_words(nbits, ncols), dtype=torch.int64, device="cuda")
    root_dev = pkg.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, 4, d_scr)
    torch.cuda.synchronize()
    host = torch.empty(N * ncols, dtype=torch.int64, pin_memory=True)
    host.copy_(d_trace)
    del d_trace, d_lde, d_tree, d_scr
    torch.cuda.empty_cache()
    lib = pkg.load()
    pkg.set_hash_family(2)
    bufs = pkg.DeviceBuffers(arity=4, n_streams=2)
    try:
        shape = pkg.StarkShape(nbits, nbe, ncols, 4)
        params = pkg.StepsParams()
        params.trace = host.data_ptr()
        root = np.zeros(4, dtype=np.uint64)
        assert lib.commit_witness(shape.ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"") < 2
        lib.get_stream_proofs(bufs.ptr)
        assert bufs.error() == 0, lib.b200_last_error()
    finally:
        bufs.close()
    assert (root == root_dev).all(), (root, root_dev)
