"""Indexed witness (instruction-table columns; unpack_indexed, starks_gpu.cu:125-185).

Each row carries an instruction index and the runtime columns; the other columns come from the
indexed table entry (an index past the table selects entry 0).  The commit must equal the
ordinary commit of the expanded trace (oracle).  The reference streaming entry point is
Poseidon1-only (set_hash_family(1), once per process), so it runs in a child process.
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


def to_dev(torch, arr):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.uint64).view(np.int64)).cuda()


def make_indexed(nbits, bits, source, index_bits, entries, seed):
    """Random indexed witness -> (expanded trace, rows, table)."""
    rng = np.random.default_rng(seed)
    n = 1 << nbits

    def vals(count, b):
        v = rng.integers(0, 1 << 63, size=count, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=count,
                                                                                              dtype=np.uint64)
        return v if b == 64 else v & np.uint64((1 << b) - 1)

    rt_cols = [c for c, x in enumerate(source) if not x]
    tb_cols = [c for c, x in enumerate(source) if x]
    table_vals = np.stack([vals(entries, bits[c]) for c in tb_cols], axis=1) if tb_cols else np.zeros((entries, 0), np.uint64)
    runtime = np.stack([vals(n, bits[c]) for c in rt_cols], axis=1) if rt_cols else np.zeros((n, 0), np.uint64)
    index = rng.integers(0, entries, size=n).astype(np.uint64)
    if index_bits and (1 << index_bits) > entries:
        index[::17] = np.uint64(min((1 << index_bits) - 1, entries + 3))  # out of range -> entry 0
    eff = np.where(index < entries, index, 0).astype(np.int64)
    trace = np.zeros((n, len(bits)), dtype=np.uint64)
    for k, c in enumerate(rt_cols):
        trace[:, c] = runtime[:, k]
    for k, c in enumerate(tb_cols):
        trace[:, c] = table_vals[eff, k]
    return trace, runtime, index, table_vals


CASES = [
    (8, 9, [8, 40, 64, 3, 17, 33], [1, 0, 1, 0, 0, 1], 5, 20),
    (10, 11, [32] * 13, [i % 3 == 0 for i in range(13)], 7, 100),
    (7, 9, [1, 2, 3, 60, 61, 62, 63, 64, 5, 9, 11, 13, 15, 20, 30, 40], [i % 2 for i in range(16)], 3, 6),
    (9, 10, [20] * 24, [1] * 24, 4, 9),      # every column from the table
    (9, 10, [20] * 24, [0] * 24, 0, 1),      # no table column, no index: a plain packed witness
]


@pytest.mark.parametrize("nbits,nbe,bits,source,index_bits,entries", CASES)
def test_indexed_commit_equals_expanded(pkg, torch_cuda, orc, nbits, nbe, bits, source, index_bits, entries):
    torch = torch_cuda
    pkg.init(0)
    trace, runtime, index, table_vals = make_indexed(nbits, bits, source, index_bits, entries, nbits + len(bits))
    rows, table = pkg.pack_indexed(runtime, index, index_bits, table_vals, bits, source)
    exp = orc.commit(trace, nbe, 4)[0]
    n, ncols = 1 << nbits, len(bits)
    d_rows, d_table = to_dev(torch, rows), to_dev(torch, table if table.size else np.zeros(1, np.uint64))
    d_lde = torch.zeros((1 << nbe) * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(pkg.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(n * ncols, dtype=torch.int64, device="cuda")
    root = pkg.commit_indexed_device(d_lde, d_tree, d_rows, rows.shape[1], d_table, entries, table.shape[1],
                                     index_bits, bits, source, nbits, nbe, 4, d_scr)
    assert (root == exp).all()
    nbytes = pkg.stream_commit_slot_bytes(nbits, nbe, ncols, rows.shape[1])
    slot = torch.full((nbytes // 8,), -1, dtype=torch.int64, device="cuda")
    root2 = pkg.stream_commit_indexed(slot, nbytes // 8, rows, bits, source, index_bits, d_table, entries,
                                      table.shape[1], nbits, nbe)
    assert (root2 == exp).all()


def test_indexed_commit_many_columns(pkg, torch_cuda, orc):
    """290 columns (half from a 9-entry table): the column bytes travel in the kernel parameters."""
    torch = torch_cuda
    pkg.init(0)
    nbits, nbe = 6, 7
    bits = [(i * 13) % 64 + 1 for i in range(290)]
    source = [i % 2 for i in range(290)]
    trace, runtime, index, table_vals = make_indexed(nbits, bits, source, 4, 9, 290)
    rows, table = pkg.pack_indexed(runtime, index, 4, table_vals, bits, source)
    d_rows, d_table = to_dev(torch, rows), to_dev(torch, table)
    n, ncols = 1 << nbits, len(bits)
    d_lde = torch.zeros((1 << nbe) * ncols, dtype=torch.int64, device="cuda")
    d_tree = torch.zeros(pkg.tree_num_elements(1 << nbe, 4), dtype=torch.int64, device="cuda")
    d_scr = torch.zeros(n * ncols, dtype=torch.int64, device="cuda")
    root = pkg.commit_indexed_device(d_lde, d_tree, d_rows, rows.shape[1], d_table, 9, table.shape[1], 4, bits,
                                     source, nbits, nbe, 4, d_scr)
    assert (root == orc.commit(trace, nbe, 4)[0]).all()


def test_indexed_rejects(pkg, torch_cuda):
    torch = torch_cuda
    pkg.init(0)
    d = torch.zeros(1 << 12, dtype=torch.int64, device="cuda")
    with pytest.raises(pkg.B200Error):  # table columns wider than words_per_entry
        pkg.commit_indexed_device(d, d, d, 1, d, 4, 1, 2, [40, 40], [1, 1], 4, 5, 4, d)
    with pytest.raises(pkg.B200Error):  # row columns + index wider than words_per_row
        pkg.commit_indexed_device(d, d, d, 1, d, 4, 1, 8, [60], [0], 4, 5, 4, d)
    with pytest.raises(pkg.B200Error):  # table columns but no entries
        pkg.commit_indexed_device(d, d, d, 1, d, 0, 1, 2, [40], [1], 4, 5, 4, d)


_CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import load_package
from test_gpu_indexed import make_indexed
import oracle
pkg = load_package()
lib = pkg.load()
pkg.set_hash_family(1)
bits = [8, 40, 64, 3, 17, 33, 12, 12, 12, 12, 12, 12, 12, 50]
source = [1, 0, 1, 0, 0, 1, 1, 0, 1, 0, 1, 0, 1, 0]
nb, nbe, ib, ent = 9, 10, 5, 20
trace, runtime, index, table_vals = make_indexed(nb, bits, source, ib, ent, 77)
rows, table = pkg.pack_indexed(runtime, index, ib, table_vals, bits, source)
bufs = pkg.DeviceBuffers(arity=4, n_streams=1)
widths = np.array(bits, dtype=np.uint64)
srcs = np.array(source, dtype=np.uint8)
root = np.zeros(4, dtype=np.uint64)
nbytes = lib.stream_commit_slot_bytes(nb, nbe, len(bits), rows.shape[1])
lib.configure_stream_commit_slots(bufs.ptr, 1, nbytes)
out = {}
assert lib.b200_register_indexed_air(bufs.ptr, 3, 4, len(bits), srcs.ctypes.data, ib) == 0
args = (rows.ctypes.data, nb, nbe, len(bits), rows.shape[1], widths.ctypes.data, root.ctypes.data)
out["no_table"] = lib.commit_witness_streaming(bufs.ptr, 0, 3, 4, *args)
tab = np.ascontiguousarray(table)
lib.register_instruction_table(bufs.ptr, 3, 4, tab.ctypes.data, ent, tab.shape[1])
out["rc"] = lib.commit_witness_streaming(bufs.ptr, 0, 3, 4, *args)
out["root_ok"] = bool((root == oracle.Oracle(family=1).commit(trace, nbe, 4)[0]).all())
bufs.close()
print(json.dumps(out))
"""


def test_reference_streaming_indexed_in_child_process(pkg, torch_cuda):
    env = dict(os.environ, PYTHONPATH=os.path.join(REPO, "tests") + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", _CHILD, REPO], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res == {"no_table": -16, "rc": 0, "root_ok": True}, res
