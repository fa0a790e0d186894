"""commit_witness on an idle device hashes in 12-column chunks while the trace's column blocks
are still crossing PCIe; with an earlier commit in flight it uses the one-pass leaf kernel.

Both orders must give the reference root (oracle: NTT_Goldilocks::LDE + the row sponge and
arity-4 tree, poseidon2_goldilocks.cpp:42-175).  Shapes are large enough (N >= 2^16, >= 128
columns) for the trace to cross in several column blocks (16, 24, 48, then 64 columns), with ragged
last blocks and chunks.
Poseidon1 runs in a child process because set_hash_family is once per process.
"""
import ctypes
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
def dev(pkg):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg.init(0)
    return pkg


def _submit(dev, lib, bufs, nb, nbe, nc, seed, keep):
    shape = dev.StarkShape(nb, nbe, nc, 4)
    trace = oracle.random_field((1 << nb, nc), seed)
    params = dev.StepsParams()
    params.trace = trace.ctypes.data
    root = np.zeros(4, dtype=np.uint64)
    sid = lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"")
    assert sid < 2, lib.b200_last_error()
    keep.append((shape, trace, params, root, nbe))


@pytest.mark.parametrize("nb,nbe,nc", [(16, 17, 130), (16, 17, 141), (16, 18, 200)])
def test_idle_then_busy_commits_match_oracle(dev, orc, nb, nbe, nc):
    lib = dev.load()
    dev.set_hash_family(2)
    bufs = dev.DeviceBuffers(arity=4, n_streams=2)
    keep = []
    try:
        _submit(dev, lib, bufs, nb, nbe, nc, 9100 + nc, keep)       # idle device: chunked sponge
        _submit(dev, lib, bufs, nb, nbe, nc + 3, 9200 + nc, keep)   # first still running: leaf kernel
        lib.get_stream_proofs(bufs.ptr)
        assert bufs.error() == 0
        for shape, trace, _, root, e in keep:
            assert (root == orc.commit(trace, e, 4)[0]).all(), trace.shape
    finally:
        bufs.close()


_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from conftest import load_package
import oracle
pkg = load_package()
lib = pkg.load()
pkg.set_hash_family(1)
bufs = pkg.DeviceBuffers(arity=4, n_streams=2)
nb, nbe, nc = 16, 17, 137
shape = pkg.StarkShape(nb, nbe, nc, 4)
trace = oracle.random_field((1 << nb, nc), 4242)
params = pkg.StepsParams()
params.trace = trace.ctypes.data
root = np.zeros(4, dtype=np.uint64)
sid = lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"")
lib.get_stream_proofs(bufs.ptr)
ok = bool((root == oracle.Oracle(family=1).commit(trace, nbe, 4)[0]).all())
err = bufs.error()
bufs.close()
print(json.dumps({"sid": int(sid), "err": int(err), "ok": ok}))
"""


def test_poseidon1_chunked_commit_in_child_process(pkg, dev):
    r = subprocess.run([sys.executable, "-c", _CHILD, REPO], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res == {"sid": 0, "err": 0, "ok": True}, res


def test_commit_witness_from_registered_host_memory(dev, orc):
    """proofman pins its trace buffers with register_host_memory (memory_handler.rs) before
    committing; the commit from a registered buffer equals the oracle's, and unregistering works."""
    import mmap
    lib = dev.load()
    dev.set_hash_family(2)
    assert lib.register_host_memory(None, 4096) == 0 and lib.register_host_memory(None, 0) == 0
    nb, nbe, nc = 16, 17, 129
    nbytes = (1 << nb) * nc * 8
    size = (nbytes + mmap.PAGESIZE - 1) // mmap.PAGESIZE * mmap.PAGESIZE
    region = mmap.mmap(-1, size)  # page-aligned anonymous memory, like a Rust Vec's pages
    trace = np.frombuffer(region, dtype=np.uint64, count=(1 << nb) * nc).reshape(1 << nb, nc)
    trace[:] = oracle.random_field((1 << nb, nc), 777)
    base = ctypes.addressof(ctypes.c_char.from_buffer(region))
    assert lib.register_host_memory(base, size) == 1
    bufs = dev.DeviceBuffers(arity=4, n_streams=2)
    try:
        shape = dev.StarkShape(nb, nbe, nc, 4)
        params = dev.StepsParams()
        params.trace = base
        root = np.zeros(4, dtype=np.uint64)
        assert lib.commit_witness(shape.setup_ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"") < 2
        lib.get_stream_proofs(bufs.ptr)
        assert bufs.error() == 0
        assert (root == orc.commit(np.array(trace), nbe, 4)[0]).all()
    finally:
        bufs.close()
        lib.unregister_host_memory(base)
