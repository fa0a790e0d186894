"""Poseidon1 (hash family 1) on the device, against the reference's Poseidon1 goldens and the oracle.

The native b200_* entry points switch family with b200_set_native_hash_family; the reference entry
points follow set_hash_family, which the reference allows once per process, so that path is run in
a child process.  Bit-exact: canonical u64 words.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture()
def p1dev(pkg, torch_cuda):
    pkg.init(0)
    pkg.set_native_hash_family(1)
    try:
        yield pkg
    finally:
        pkg.set_native_hash_family(2)


@pytest.fixture(scope="module")
def orc1():
    return oracle.Oracle(family=1)


def to_dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint64).view(np.int64)).cuda()


def from_dev(t):
    return t.cpu().numpy().view(np.uint64)


def _fib(n):
    out = [0, 1]
    while len(out) < n:
        out.append((out[-1] + out[-2]) % oracle.P)
    return np.array(out[:n], dtype=np.uint64)


def _permute(dev, torch, states, w):
    x = to_dev(torch, states)
    y = torch.zeros_like(x)
    dev.permute_device(y, x, states.shape[0], w)
    torch.cuda.synchronize()
    return from_dev(y).reshape(states.shape)


def test_p1_permute_goldens(p1dev, torch_cuda, kats):
    g = kats["poseidon1"]
    torch = torch_cuda
    assert [int(v) for v in _permute(p1dev, torch, _fib(12)[None], 12)[0]] == g["PERMUTE_FIB_W12_GOLDEN"]
    assert [int(v) for v in _permute(p1dev, torch, np.zeros((1, 12), np.uint64), 12)[0]] == g["PERMUTE_ZERO_W12_GOLDEN"]
    assert [int(v) for v in _permute(p1dev, torch, np.arange(8, dtype=np.uint64)[None], 8)[0]] == \
        g["PERMUTE_W8_POSEIDON1_PLONKY3_GOLDEN"]
    assert [int(v) for v in _permute(p1dev, torch, np.arange(16, dtype=np.uint64)[None], 16)[0]] == \
        g["PERMUTE_W16_POSEIDON1_GOLDEN"]


@pytest.mark.parametrize("w", [8, 12, 16])
def test_p1_permute_random_vs_oracle(p1dev, torch_cuda, orc1, w):
    x = oracle.random_field((700, w), 300 + w)
    x[:4] = np.uint64(0xFFFFFFFFFFFFFFFF)  # loose inputs are taken mod p
    x[4:8] = np.uint64(oracle.P - 1)
    y = _permute(p1dev, torch_cuda, x, w)
    for i in range(0, 700, 37):
        assert (y[i] == orc1.permute(x[i])).all(), i
    for i in range(8):
        assert (y[i] == orc1.permute(x[i])).all(), i


def test_p1_seeded_commits(p1dev, torch_cuda, kats):
    torch = torch_cuda
    for case in kats["seeded_commits_poseidon1"]:
        nb, nbe, nc, ar = case["nBits"], case["nBitsExt"], case["nCols"], case["arity"]
        trace = oracle.random_field((1 << nb, nc), case["seed"])
        d_trace = to_dev(torch, trace)
        d_lde = torch.zeros((1 << nbe) * nc, dtype=torch.int64, device="cuda")
        d_tree = torch.zeros(p1dev.tree_num_elements(1 << nbe, ar), dtype=torch.int64, device="cuda")
        d_scr = torch.zeros(p1dev.lde_scratch_words(nb, nc), dtype=torch.int64, device="cuda")
        root = p1dev.commit_device(d_lde, d_tree, d_trace, nb, nbe, nc, ar, d_scr)
        assert [int(v) for v in root] == case["root"], case


@pytest.mark.parametrize("nrows,ncols,arity", [(64, 0, 2), (100, 9, 2), (256, 13, 3), (1000, 25, 4), (1, 5, 4)])
def test_p1_merkletree_vs_oracle(p1dev, torch_cuda, orc1, nrows, ncols, arity):
    torch = torch_cuda
    m = oracle.random_field((nrows, ncols), nrows + ncols)
    d_src = to_dev(torch, m.T.copy() if ncols else np.zeros(1, np.uint64))
    d_tree = torch.zeros(p1dev.tree_num_elements(nrows, arity), dtype=torch.int64, device="cuda")
    p1dev.merkletree_device(d_tree, d_src, 1, nrows, ncols, nrows, arity)
    torch.cuda.synchronize()
    assert (from_dev(d_tree) == orc1.merkletree(m, arity)).all()


def test_p1_queries_hash_to_root(p1dev, torch_cuda, orc1):
    torch = torch_cuda
    nb, nbe, nc, ar = 8, 9, 11, 4
    trace = oracle.random_field((1 << nb, nc), 77)
    d_trace = to_dev(torch, trace)
    d_lde = torch.zeros((1 << nbe) * nc, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(p1dev.tree_num_elements(1 << nbe, ar), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(p1dev.lde_scratch_words(nb, nc), dtype=torch.int64, device="cuda")
    root = p1dev.commit_device(d_lde, d_tree, d_trace, nb, nbe, nc, ar, d_scr)
    rows = np.array([0, 5, 511, 300], dtype=np.uint64)
    words = p1dev.query_proof_words(1 << nbe, nc, ar)
    d_out = torch.zeros(len(rows) * words, dtype=torch.int64, device="cuda")
    p1dev.query_openings_device(d_out, d_lde, 1 << nbe, nc, d_tree, ar, to_dev(torch, rows), len(rows))
    torch.cuda.synchronize()
    out = from_dev(d_out).reshape(len(rows), words)
    for i, r in enumerate(rows):
        assert (orc1.root_from_proof(out[i], nc, 1 << nbe, ar, int(r)) == root).all()


def test_p1_batch_and_server(p1dev, torch_cuda, orc1):
    """The batched plan and the commit server hash with the family they were created under."""
    torch = torch_cuda
    lib = p1dev.load()
    shapes = [(8, 9, 13), (10, 11, 5), (9, 11, 30), (6, 7, 1)]
    traces = [oracle.random_field((1 << nb, nc), 500 + i) for i, (nb, nbe, nc) in enumerate(shapes)]
    exp = [orc1.commit(t, nbe, 4)[0] for t, (nb, nbe, nc) in zip(traces, shapes)]
    keep = []
    descs = (p1dev.BatchInstance * len(shapes))()
    for i, ((nb, nbe, nc), t) in enumerate(zip(shapes, traces)):
        bufs = [to_dev(torch, t), torch.zeros((1 << nb) * nc, dtype=torch.int64, device="cuda"),
                torch.zeros((1 << nbe) * nc, dtype=torch.int64, device="cuda"),
                torch.zeros(p1dev.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device="cuda")]
        keep.append(bufs)
        d = descs[i]
        d.d_trace, d.d_scratch, d.d_lde, d.d_tree = [b.data_ptr() for b in bufs]
        d.nBits, d.nBitsExt, d.nCols, d.arity = nb, nbe, nc, 4
    roots = np.zeros((len(shapes), 4), dtype=np.uint64)
    assert lib.b200_commit_batch_device(descs, len(shapes), roots.ctypes.data, None) == 0, lib.b200_last_error()
    for i in range(len(shapes)):
        assert (roots[i] == exp[i]).all(), i
    srv = lib.b200_server_new(0, 1 << 30, 2)
    assert srv
    try:
        outs = [np.zeros(4, dtype=np.uint64) for _ in shapes]
        ids = [lib.b200_server_submit(srv, t.ctypes.data, nb, nbe, nc, 4, o.ctypes.data)
               for t, (nb, nbe, nc), o in zip(traces, shapes, outs)]
        assert all(i > 0 for i in ids)
        assert lib.b200_server_wait_all(srv, 60000) == 0
        for o, e in zip(outs, exp):
            assert (o == e).all()
    finally:
        lib.b200_server_free(srv)


_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import load_package
import oracle
pkg = load_package()
lib = pkg.load()
pkg.set_hash_family(1)
out = {}
for nb, nbe, nc, ar in ((6, 7, 5, 4), (7, 9, 12, 3), (5, 6, 3, 2)):
    trace = oracle.random_field((1 << nb, nc), 900 + nb)
    root = np.zeros(4, dtype=np.uint64)
    lib.write_custom_commit(root.ctypes.data, ar, nb, nbe, nc, None, trace.ctypes.data, None)
    exp = oracle.Oracle(family=1).commit(trace, nbe, ar)[0]
    out["%d_%d_%d_%d" % (nb, nbe, nc, ar)] = bool((root == exp).all())
print(json.dumps(out))
"""


def test_p1_reference_abi_in_child_process(pkg, torch_cuda):
    r = subprocess.run([sys.executable, "-c", _CHILD, REPO], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res and all(res.values()), res
