"""Streaming slot commit of a bit-packed witness (commit_witness_streaming / streamCommitPacked).

The root must equal the ordinary commit of the unpacked trace (oracle, same hash family): the
chunked absorb is the row sponge block by block.  The reference entry points are Poseidon1-only
and need set_hash_family(1), which is set once per process, so they run in a child process;
the native form runs here under both families.
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


def _packed_trace(nbits, bits, seed):
    rng = np.random.default_rng(seed)
    n = 1 << nbits
    trace = np.zeros((n, len(bits)), dtype=np.uint64)
    for c, b in enumerate(bits):
        v = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
        trace[:, c] = v if b == 64 else v & np.uint64((1 << b) - 1)
    return trace


@pytest.mark.parametrize("family", [1, 2])
@pytest.mark.parametrize("nbits,nbe,bits", [
    (6, 7, [17]), (8, 9, [3] * 12), (8, 10, [64, 1, 33, 31, 2, 64, 17, 5, 9, 9, 9, 40, 63]),
    (10, 11, [32] * 30), (7, 9, [(7 * i) % 64 + 1 for i in range(64)])])
def test_stream_commit_equals_ordinary_commit(pkg, torch_cuda, family, nbits, nbe, bits):
    torch = torch_cuda
    pkg.init(0)
    pkg.set_native_hash_family(family)
    try:
        trace = _packed_trace(nbits, bits, nbits * 100 + len(bits))
        packed = pkg.pack_rows(trace, bits)
        nbytes = pkg.stream_commit_slot_bytes(nbits, nbe, len(bits), packed.shape[1])
        assert nbytes > 0
        slot = torch.full((nbytes // 8,), -1, dtype=torch.int64, device="cuda")  # poisoned slot
        root = pkg.stream_commit_packed(slot, nbytes // 8, packed, bits, nbits, nbe)
        exp = oracle.Oracle(family=family).commit(trace, nbe, 4)[0]
        assert (root == exp).all()
        root2 = pkg.stream_commit_packed(slot, nbytes // 8, packed, bits, nbits, nbe)  # slot reuse
        assert (root2 == exp).all()
    finally:
        pkg.set_native_hash_family(2)


def test_stream_commit_rejects(pkg, torch_cuda):
    torch = torch_cuda
    pkg.init(0)
    lib = pkg.load()
    assert pkg.stream_commit_slot_bytes(8, 9, 0, 1) == 0       # no columns
    assert pkg.stream_commit_slot_bytes(8, 9, 65, 70) == 0     # wider than the slot layout
    assert pkg.stream_commit_slot_bytes(8, 8, 4, 1) == 0       # no extension
    bits = [30, 30, 30]
    trace = _packed_trace(6, bits, 1)
    packed = pkg.pack_rows(trace, bits)
    nbytes = pkg.stream_commit_slot_bytes(6, 7, 3, packed.shape[1])
    small = torch.zeros(nbytes // 16, dtype=torch.int64, device="cuda")
    with pytest.raises(pkg.B200Error):
        pkg.stream_commit_packed(small, nbytes // 16, packed, bits, 6, 7)
    slot = torch.zeros(nbytes // 8, dtype=torch.int64, device="cuda")
    with pytest.raises(pkg.B200Error):  # 158 bits of widths do not fit the 2 packed words per row
        pkg.stream_commit_packed(slot, nbytes // 8, packed, [64, 64, 30], 6, 7)
    # the reference entry refuses a Poseidon2 process (this test process uses family 2)
    pkg.set_hash_family(2)
    bufs = pkg.DeviceBuffers(arity=4, n_streams=1)
    try:
        widths = np.array(bits, dtype=np.uint64)
        root = np.zeros(4, dtype=np.uint64)
        assert lib.commit_witness_streaming(bufs.ptr, 0, 0, 0, packed.ctypes.data, 6, 7, 3, packed.shape[1],
                                            widths.ctypes.data, root.ctypes.data) == -11  # no slots yet
        lib.configure_stream_commit_slots(bufs.ptr, 1, nbytes)
        assert lib.get_stream_commit_slots(bufs.ptr) == 1
        assert lib.commit_witness_streaming(bufs.ptr, 0, 0, 0, packed.ctypes.data, 6, 7, 3, packed.shape[1],
                                            widths.ctypes.data, root.ctypes.data) == -15  # not Poseidon1
    finally:
        bufs.close()


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
bufs = pkg.DeviceBuffers(arity=4, n_streams=1)
out = {}
bits = [21, 64, 7, 33, 12, 12, 50, 1, 2, 3, 60, 44, 5, 6]
rng = np.random.default_rng(3)
nb, nbe = 9, 10
trace = np.zeros((1 << nb, len(bits)), dtype=np.uint64)
for c, b in enumerate(bits):
    v = rng.integers(0, 1 << 63, size=1 << nb, dtype=np.uint64) * np.uint64(2)
    trace[:, c] = v if b == 64 else v & np.uint64((1 << b) - 1)
packed = pkg.pack_rows(trace, bits)
widths = np.array(bits, dtype=np.uint64)
nbytes = lib.stream_commit_slot_bytes(nb, nbe, len(bits), packed.shape[1])
lib.configure_stream_commit_slots(bufs.ptr, 2, nbytes)
root = np.zeros(4, dtype=np.uint64)
args = (nb, nbe, len(bits), packed.shape[1], widths.ctypes.data, root.ctypes.data)
out["rc0"] = lib.commit_witness_streaming(bufs.ptr, 0, 0, 0, packed.ctypes.data, *args)
out["root_ok"] = bool((root == oracle.Oracle(family=1).commit(trace, nbe, 4)[0]).all())
root[:] = 0
out["rc1"] = lib.commit_witness_streaming(bufs.ptr, 1, 0, 0, packed.ctypes.data, *args)
out["root1_ok"] = bool((root == oracle.Oracle(family=1).commit(trace, nbe, 4)[0]).all())
out["bad_slot"] = lib.commit_witness_streaming(bufs.ptr, 2, 0, 0, packed.ctypes.data, *args)
out["too_small"] = lib.commit_witness_streaming(bufs.ptr, 0, 0, 0, packed.ctypes.data, nb + 1, nbe + 1, len(bits),
                                                packed.shape[1], widths.ctypes.data, root.ctypes.data)
lib.stream_commit_pause()
out["paused"] = lib.commit_witness_streaming(bufs.ptr, 0, 0, 0, packed.ctypes.data, *args)
bufs.close()
print(json.dumps(out))
"""


def test_reference_streaming_entry_in_child_process(pkg, torch_cuda):
    r = subprocess.run([sys.executable, "-c", _CHILD, REPO], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res == {"rc0": 0, "root_ok": True, "rc1": 0, "root1_ok": True, "bad_slot": -12, "too_small": -13,
                   "paused": -14}, res
