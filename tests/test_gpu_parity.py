"""Bit-exact parity of the CUDA commit path against the reference's known answers and the oracle.

Every call goes through the C-ABI library (libpil2_b200.so); torch only allocates device memory.
Tolerance: none — integer field arithmetic, results compared as canonical u64 words.
"""
import hashlib
import os
import tempfile

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

P = oracle.P


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


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


@pytest.mark.parametrize("w", [8, 12, 16])
def test_permute_golden(dev, torch_cuda, kats, w):
    x = to_dev(torch_cuda, np.arange(w, dtype=np.uint64))
    y = torch_cuda.zeros_like(x)
    dev.permute_device(y, x, 1, w)
    torch_cuda.cuda.synchronize()
    assert [int(v) for v in from_dev(y)] == kats["poseidon2"]["PERMUTE_W%d_GOLDEN" % w]


@pytest.mark.parametrize("w", [8, 12, 16])
def test_permute_random_vs_oracle(dev, torch_cuda, orc, w):
    n = 1000
    x = oracle.random_field((n, w), 77 + w)
    # loose (non-canonical) inputs are taken mod p
    x[:5] = np.uint64(0xFFFFFFFFFFFFFFFF)
    y = torch_cuda.zeros((n * w,), dtype=torch_cuda.int64, device="cuda")
    dev.permute_device(y, to_dev(torch_cuda, x.reshape(-1)), n, w)
    got = from_dev(y).reshape(n, w)
    for i in range(0, n, 97):
        assert (got[i] == orc.permute(x[i])).all()
    assert (got[:5] == orc.permute(x[0])).all()


@pytest.mark.parametrize("arity", [2, 3, 4])
def test_linear_hash_golden_single_row(dev, torch_cuda, kats, arity):
    # a 1-row tree's root is the row's linear hash (test_poseidon2_cpu.cpp:418-442)
    w = 4 * arity
    row = to_dev(torch_cuda, np.arange(1, 21, dtype=np.uint64))
    tree = torch_cuda.zeros((4,), dtype=torch_cuda.int64, device="cuda")
    dev.merkletree_device(tree, row, 20, 1, 20, 1, arity)
    assert [int(v) for v in from_dev(tree)] == kats["poseidon2"]["LINEAR_HASH_W%d_GOLDEN" % w]


def test_lde_block_golden(dev, kats):
    n, ncols = 16, 8
    a = np.zeros((n, ncols), dtype=np.uint64)
    for j in range(ncols):
        a[0, j] = a[1, j] = 1 + j
    for i in range(2, n):
        a[i] = (a[i - 1] + a[i - 2]) % np.uint64(P)
    _, lde, _ = dev.commit_host(a, 5, 4, want_lde=True)
    assert [int(v) for v in lde[0]] == kats["lde_block_16_32_col0"]


def test_seeded_reference_commits(dev, kats):
    """Roots, LDEs and full trees of the reference CPU build on seeded inputs."""
    for c in kats["seeded_commits"]:
        trace = oracle.random_field((1 << c["nBits"], c["nCols"]), c["seed"])
        root, lde, tree = dev.commit_host(trace, c["nBitsExt"], c["arity"], want_lde=True, want_tree=True)
        assert [int(v) for v in root] == c["root"], c
        assert digest(lde.T) == c["lde_sha256"], c
        assert digest(tree) == c["tree_sha256"], c


SHAPES = [  # (nBits, nBitsExt, nCols, arity)
    (1, 3, 1, 4), (2, 3, 4, 4), (3, 5, 2, 2), (5, 6, 13, 4), (7, 8, 12, 4), (7, 9, 24, 3), (9, 10, 11, 2),
    (11, 12, 5, 4), (12, 13, 3, 4), (12, 14, 17, 4), (13, 14, 9, 3), (14, 15, 16, 4), (14, 16, 3, 4),
    (15, 16, 7, 4), (6, 6, 5, 4), (0, 3, 3, 4), (4, 8, 2, 4),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_commit_vs_oracle(dev, orc, shape):
    nb, nbe, nc, ar = shape
    trace = oracle.random_field((1 << nb, nc), 1000 + nb * 37 + nbe * 5 + nc)
    root, lde, tree = dev.commit_host(trace, nbe, ar, want_lde=True, want_tree=True)
    r2, l2, t2 = orc.commit(trace, nbe, ar)
    assert (lde.T == l2).all()
    assert (tree == t2).all()
    assert (root == r2).all()


def test_noncanonical_trace_taken_mod_p(dev, orc):
    trace = oracle.random_field((1 << 8, 6), 4242)
    trace[::3] %= np.uint64(2**32 - 1)  # small words, which have a second 64-bit representative
    loose = trace.copy()
    small = trace < np.uint64(2**32 - 1)
    loose[small] += np.uint64(P)  # same field elements, non-canonical words
    r1, l1, _ = dev.commit_host(trace, 9, 4, want_lde=True)
    r2, l2, _ = dev.commit_host(loose, 9, 4, want_lde=True)
    assert small.any()
    assert (r1 == r2).all() and (l1 == l2).all()


def test_zero_columns_gives_zero_digests(dev, orc):
    trace = np.zeros((1 << 5, 0), dtype=np.uint64)
    root, _, tree = dev.commit_host(trace, 6, 4, want_tree=True)
    r2, _, t2 = orc.commit(trace, 6, 4)
    assert (tree == t2).all() and (root == r2).all()


def test_c1_config_root(dev, kats):
    """The CPU-runnable single-AIR case: 2^16 x 32, blowup 2, arity 4 and 3."""
    for c in kats["seeded_commits"]:
        if c["nBits"] == 16:
            trace = oracle.random_field((1 << 16, 32), c["seed"])
            root, _, _ = dev.commit_host(trace, 17, c["arity"])
            assert [int(v) for v in root] == c["root"]


def test_device_api_column_major_input(dev, torch_cuda, orc):
    nb, nbe, nc, ar = 12, 13, 20, 4
    trace = oracle.random_field((1 << nb, nc), 31337)
    d_trace_cm = to_dev(torch_cuda, trace.T.copy().reshape(-1))
    n, next_ = 1 << nb, 1 << nbe
    d_lde = torch_cuda.zeros((nc * next_,), dtype=torch_cuda.int64, device="cuda")
    d_tree = torch_cuda.zeros((dev.tree_num_elements(next_, ar),), dtype=torch_cuda.int64, device="cuda")
    d_scr = torch_cuda.zeros((dev.lde_scratch_words(nb, nc),), dtype=torch_cuda.int64, device="cuda")
    root = dev.commit_device(d_lde, d_tree, d_trace_cm, nb, nbe, nc, ar, d_scr, trace_rowmajor=False)
    r2, l2, t2 = orc.commit(trace, nbe, ar)
    assert (root == r2).all()
    assert (from_dev(d_lde).reshape(nc, next_).T == l2).all()
    # the column-major input is left untouched
    assert (from_dev(d_trace_cm).reshape(nc, n).T == trace).all()


def test_lde_rows_query(dev, torch_cuda, orc):
    nb, nbe, nc = 10, 12, 9
    trace = oracle.random_field((1 << nb, nc), 99)
    _, lde, _ = dev.commit_host(trace, nbe, 4, want_lde=True)
    d_lde = to_dev(torch_cuda, lde.reshape(-1))
    rows = np.array([0, 5, 4095, 1234, 77], dtype=np.uint64)
    d_rows = to_dev(torch_cuda, rows)
    out = torch_cuda.zeros((rows.size * nc,), dtype=torch_cuda.int64, device="cuda")
    dev.lde_rows_device(out, d_lde, 1 << nbe, nc, d_rows, rows.size)
    assert (from_dev(out).reshape(rows.size, nc) == lde.T[rows.astype(np.int64)]).all()


def test_fill_random_host_device_agree(dev, torch_cuda):
    n = 100003
    d = torch_cuda.zeros((n,), dtype=torch_cuda.int64, device="cuda")
    dev.fill_random_device(d, n, 5)
    h = dev.fill_random_host(n, 5)
    assert (from_dev(d) == h).all()
    assert (h < np.uint64(P)).all()


def test_determinism_and_poisoned_buffers(dev, torch_cuda, orc):
    """Outputs do not depend on stale buffer contents (0xAB fill, as test_ntt_gpu.cu:379)."""
    nb, nbe, nc, ar = 13, 14, 15, 4
    trace = oracle.random_field((1 << nb, nc), 2024)
    next_ = 1 << nbe
    roots = []
    for fill in (0, 0xABABABABABABABAB - 2**64):
        d_trace = to_dev(torch_cuda, trace.reshape(-1))
        d_lde = torch_cuda.full((nc * next_,), fill, dtype=torch_cuda.int64, device="cuda")
        d_tree = torch_cuda.full((dev.tree_num_elements(next_, ar),), fill, dtype=torch_cuda.int64, device="cuda")
        d_scr = torch_cuda.full((dev.lde_scratch_words(nb, nc),), fill, dtype=torch_cuda.int64, device="cuda")
        roots.append(dev.commit_device(d_lde, d_tree, d_trace, nb, nbe, nc, ar, d_scr))
    assert (roots[0] == roots[1]).all()
    assert (roots[0] == orc.commit(trace, nbe, ar)[0]).all()


# ---------------------------------------------------------------- reference ABI ----

def test_commit_witness_async_pool(dev, orc):
    lib = dev.load()
    dev.set_hash_family(2)
    bufs = dev.DeviceBuffers(arity=4, n_streams=2)
    shapes = [(10, 11, 7), (12, 13, 20), (9, 11, 3), (11, 12, 31), (8, 9, 1)]
    keep = []
    roots = []
    for i, (nb, nbe, nc) in enumerate(shapes):
        shape = dev.StarkShape(nb, nbe, nc, 4)
        trace = oracle.random_field((1 << nb, nc), 600 + i)
        params = dev.StepsParams()
        params.trace = trace.ctypes.data
        root = np.zeros(4, dtype=np.uint64)
        sid = lib.commit_witness(shape.setup_ptr, ctypes_ref(params), i, 0, 0, root.ctypes.data, bufs.ptr, b"")
        assert sid < 2, dev.load().b200_last_error()
        keep.append((shape, trace, params))
        roots.append(root)
    lib.get_stream_proofs(bufs.ptr)
    assert bufs.error() == 0
    for (shape, trace, _), root in zip(keep, roots):
        assert (root == orc.commit(trace, shape.nbits_ext, 4)[0]).all()
    bufs.close()


def ctypes_ref(s):
    import ctypes
    return ctypes.addressof(s)


def test_write_custom_commit_file(dev, orc):
    lib = dev.load()
    dev.set_hash_family(2)
    nb, nbe, nc, ar = 9, 10, 6, 4
    trace = oracle.random_field((1 << nb, nc), 8080)
    root = np.zeros(4, dtype=np.uint64)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "custom.bin").encode()
        lib.write_custom_commit(root.ctypes.data, ar, nb, nbe, nc, None, trace.ctypes.data, path)
        blob = np.fromfile(path.decode(), dtype=np.uint64)
    r2, l2, t2 = orc.commit(trace, nbe, ar)
    n, next_ = 1 << nb, 1 << nbe
    assert (root == r2).all()
    assert (blob[:4] == r2).all()
    assert (blob[4:4 + n * nc].reshape(nc, n).T == trace).all()
    off = 4 + n * nc
    assert (blob[off:off + next_ * nc].reshape(nc, next_).T == l2).all()
    assert (blob[off + next_ * nc:] == t2).all()


def test_calculate_const_tree_layout(dev, orc):
    lib = dev.load()
    dev.set_hash_family(2)
    nb, nbe, nc, ar = 8, 10, 5, 3
    shape = dev.StarkShape(nb, nbe, nc, ar)
    pols = oracle.random_field((1 << nb, nc), 123)
    size = int(lib.get_const_tree_size(shape.ptr))
    out = np.zeros(size, dtype=np.uint64)
    lib.calculate_const_tree(shape.ptr, pols.ctypes.data, out.ctypes.data, None)
    r2, l2, t2 = orc.commit(pols, nbe, ar)
    next_ = 1 << nbe
    assert (out[:next_ * nc].reshape(nc, next_).T == l2).all()
    assert (out[next_ * nc:] == t2).all()


def test_bad_shapes_rejected(dev):
    with pytest.raises(dev.B200Error):
        dev.commit_host(np.zeros((4, 2), dtype=np.uint64), 1, 4)  # nBitsExt < nBits
    with pytest.raises(dev.B200Error):
        dev.commit_host(np.zeros((4, 2), dtype=np.uint64), 3, 5)  # arity 5
    with pytest.raises(dev.B200Error):
        dev.commit_host(np.zeros((4, 2), dtype=np.uint64), 27, 4)  # above 2^26 rows
