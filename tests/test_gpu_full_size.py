"""Parity at the workloads' full row counts (C2: 2^22 -> 2^23 rows at blowup 2; C4: 2^20 -> 2^22
at blowup 4), where the NTT runs its largest windows and the tree its deepest levels.

* Bit-exact against the oracle (NTT_Goldilocks::LDE, ntt_goldilocks.cpp:369-404, and the
  Poseidon2 row sponge and arity-4 tree, poseidon2_goldilocks.cpp:42-175) for a few columns:
  root, every LDE word and every tree node.
* A size-independent property for many columns: the LDE is linear, LDE(x + y) = LDE(x) + LDE(y)
  (mod p), checked word for word.
* At the full C2 (2^22 x 256, blowup 2) and C4 (2^20 x 780, blowup 4) shapes, every column:
  the one-pass device commit and the reference-facing commit_witness path against the reference's
  own CPU build run on the same seeded trace (tests/golden/full_size.json, written by
  make_full_size.py): root, the SHA-256 of the whole tree buffer, and sampled LDE rows.  The C2
  trace is also committed with Poseidon1 (hash family 1, PoseidonGoldilocks<16>::merkletree).
Calls go through the C-ABI library; torch only allocates device memory.
"""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

P = np.uint64(oracle.P)
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


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


def _full_size_fixtures():
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "full_size.json")
    with open(path) as f:
        return json.load(f)["shapes"]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.mark.parametrize("fx", _full_size_fixtures(), ids=lambda fx: fx["name"])
def test_full_size_matches_reference_cpu(dev, fx):
    """The full workload shapes, every column, against the reference CPU build's commit of the same
    seeded trace (NTT_Goldilocks::LDE + Poseidon2Goldilocks<16>::merkletree, or
    PoseidonGoldilocks<16>::merkletree for the family-1 record, run by
    make_full_size.py): the one-pass device commit (root, the whole tree buffer by SHA-256, sampled
    LDE rows word for word), then commit_witness from pinned host memory (column blocks of 16, 24,
    48, then 64, crossing PCIe while earlier blocks are extended; the sponge absorbed in 12-column
    chunks on the idle device) to the same root."""
    pkg, torch = dev
    nbits, nbe, ncols, arity = fx["nBits"], fx["nBitsExt"], fx["nCols"], fx["arity"]
    family = fx.get("family", 2)
    N, NExt = 1 << nbits, 1 << nbe
    want_root = np.array(fx["root"], dtype=np.uint64)
    d_trace = torch.empty(N * ncols, dtype=torch.int64, device="cuda")
    pkg.fill_random_device(d_trace, N * ncols, fx["seed"])
    d_lde = torch.empty(NExt * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.empty(pkg.tree_num_elements(NExt, arity), dtype=torch.int64, device="cuda")
    d_scr = torch.empty(pkg.lde_scratch_words(nbits, ncols), dtype=torch.int64, device="cuda")
    pkg.set_native_hash_family(family)
    try:
        root_dev = pkg.commit_device(d_lde, d_tree, d_trace, nbits, nbe, ncols, arity, d_scr)
        torch.cuda.synchronize()
    finally:
        pkg.set_native_hash_family(2)
    assert (root_dev == want_root).all(), ([hex(int(v)) for v in root_dev], [hex(v) for v in fx["root"]])
    tree = d_tree.cpu().numpy().view(np.uint64)
    assert tree.size == fx["tree_words"]
    assert _sha(tree) == fx["tree_sha256"]
    rows = torch.tensor(fx["sample_rows"], dtype=torch.int64, device="cuda")
    d_rows_out = torch.empty(len(fx["sample_rows"]) * ncols, dtype=torch.int64, device="cuda")
    pkg.lde_rows_device(d_rows_out, d_lde, NExt, ncols, rows, len(fx["sample_rows"]))
    block = d_rows_out.cpu().numpy().view(np.uint64).reshape(-1, ncols)
    assert [int(v) for v in block[0]] == fx["sample_row0"]
    assert _sha(block) == fx["sample_rows_sha256"]
    del d_lde, d_tree, d_scr, d_rows_out
    if family != 2:
        # the reference entry points take set_hash_family once per process: Poseidon1 runs in a child
        del d_trace
        torch.cuda.empty_cache()
        r = subprocess.run([sys.executable, "-c", _WITNESS_CHILD, REPO, str(nbits), str(nbe), str(ncols), str(arity),
                            str(fx["seed"]), str(family)], capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        root = np.array(json.loads(r.stdout.strip().splitlines()[-1])["root"], dtype=np.uint64)
    else:
        host = torch.empty(N * ncols, dtype=torch.int64, pin_memory=True)
        host.copy_(d_trace)
        del d_trace
        torch.cuda.empty_cache()
        pkg.set_hash_family(2)
        root = _commit_witness(pkg, host.data_ptr(), nbits, nbe, ncols, arity)
    assert (root == want_root).all(), (root, want_root)


def _commit_witness(pkg, host_ptr, nbits, nbe, ncols, arity):
    """commit_witness through a StarkShape setup from a pinned host trace, on two streams"""
    import ctypes
    lib = pkg.load()
    bufs = pkg.DeviceBuffers(arity=arity, n_streams=2)
    try:
        shape = pkg.StarkShape(nbits, nbe, ncols, arity)
        params = pkg.StepsParams()
        params.trace = host_ptr
        root = np.zeros(4, dtype=np.uint64)
        assert lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"") < 2
        lib.get_stream_proofs(bufs.ptr)
        assert bufs.error() == 0, lib.b200_last_error()
    finally:
        bufs.close()
    return root


_WITNESS_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import torch
from conftest import load_package
from test_gpu_full_size import _commit_witness
nbits, nbe, ncols, arity, seed, family = map(int, sys.argv[2:8])
pkg = load_package()
pkg.init(0)
pkg.set_hash_family(family)
host = torch.empty((1 << nbits) * ncols, dtype=torch.int64, pin_memory=True)
pkg.load().b200_fill_random_host(host.data_ptr(), host.numel(), seed)
root = _commit_witness(pkg, host.data_ptr(), nbits, nbe, ncols, arity)
print(json.dumps({"root": [int(v) for v in root]}))
"""
