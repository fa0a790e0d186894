"""The reference-facing commit through a starkinfo file, as proofman drives it.

proofman builds `SetupC {p_stark_info, p_expressions_bin}` with p_stark_info = stark_info_new(file, ...)
(common/src/setup.rs:45-57,206-215) and passes its address as pSetupCtx to commit_witness
(ffi_starks.rs:705-730).  Here the same calls go through ctypes; the root must equal the oracle's, and
the stream's prover buffer must hold the commit where the reference's later stages read it
(commit_witness_gpu, starks_api.cu:1599-1795): the column-major trace at mapOffsets[("cm1", false)],
the LDE at ("cm1", true) and the tree at ("mt1", true).  Large traces cross in column blocks staged at
the top of the ("cm1", true) region, so the shapes include pipelined ones at blowup 2 and 4.
"""
import ctypes
import json
import os
import tempfile

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
    pkg.set_hash_family(2)
    return pkg, torch


def write_setup(nbits, nbits_ext, ncm1, arity=4, nconst=5):
    s = {
        "starkStruct": {"nBits": nbits, "nBitsExt": nbits_ext, "nQueries": 16, "verificationHashType": "GL",
                        "merkleTreeArity": arity, "transcriptArity": arity, "merkleTreeCustom": False,
                        "lastLevelVerification": 2, "powBits": 0,
                        "steps": [{"nBits": nbits_ext}, {"nBits": max(1, nbits_ext - 4)}]},
        "nPublics": 2, "nConstants": nconst, "nStages": 2, "qDeg": 2, "qDim": 3, "nConstraints": 1,
        "customCommits": [], "openingPoints": [0, 1], "boundaries": [{"name": "everyRow"}],
        "challengesMap": [{"stage": 2}] * 3, "airgroupValuesMap": [], "airValuesMap": [{"stage": 1}],
        "proofValuesMap": [], "evMap": [{"type": "cm"}] * 9,
        "mapSectionsN": {"const": nconst, "cm1": ncm1, "cm2": 3, "cm3": 6},
    }
    d = tempfile.mkdtemp()
    path = os.path.join(d, "air.starkinfo.json")
    with open(path, "w") as f:
        json.dump(s, f)
    return path


_cudart = None


def device_words(torch, ptr, offset, n):
    """n words of device memory at ptr + 8*offset, copied to the host with the CUDA runtime's
    cudaMemcpy (device to host)."""
    global _cudart
    if _cudart is None:
        import nvidia.cuda_runtime
        base = list(nvidia.cuda_runtime.__path__)[0]
        _cudart = ctypes.CDLL(os.path.join(base, "lib", "libcudart.so.12"))
        _cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        _cudart.cudaMemcpy.restype = ctypes.c_int
    out = np.empty(n, dtype=np.uint64)
    torch.cuda.synchronize()
    assert _cudart.cudaMemcpy(out.ctypes.data, ptr + 8 * offset, 8 * n, 2) == 0  # cudaMemcpyDeviceToHost
    return out


@pytest.mark.parametrize("nbits,nbe,ncm1,arity", [(10, 11, 7, 4), (9, 11, 5, 2), (12, 13, 13, 3),
                                                  (16, 17, 200, 4), (16, 18, 130, 4)])
def test_commit_witness_from_starkinfo(dev, orc, nbits, nbe, ncm1, arity):
    pkg, torch = dev
    si = pkg.StarkInfo(write_setup(nbits, nbe, ncm1, arity))
    N, NExt = 1 << nbits, 1 << nbe
    trace = oracle.random_field((N, ncm1), 900 + nbits + ncm1)
    host = torch.from_numpy(trace.view(np.int64).copy()).pin_memory()
    params = pkg.StepsParams()
    params.trace = host.data_ptr()
    lib = pkg.load()
    bufs = pkg.DeviceBuffers(arity=arity, n_streams=2)
    try:
        root = np.zeros(4, dtype=np.uint64)
        sid = lib.commit_witness(si.setup_ptr, ctypes.addressof(params), 0, 0, 0, root.ctypes.data, bufs.ptr, b"")
        assert sid < 2, lib.b200_last_error()
        lib.get_stream_proofs(bufs.ptr)
        assert bufs.error() == 0, lib.b200_last_error()
        r_o, lde_o, tree_o = orc.commit(trace, nbe, arity)
        assert (root == r_o).all()
        aux, words = bufs.aux(sid)
        assert words >= si.offset("cm1", False) + N * ncm1
        lde = device_words(torch, aux, si.offset("cm1", True), NExt * ncm1).reshape(ncm1, NExt)
        assert (lde.T == lde_o).all()
        tree = device_words(torch, aux, si.offset("mt1", True), pkg.tree_num_elements(NExt, arity))
        assert (tree == tree_o).all()
        cm1 = device_words(torch, aux, si.offset("cm1", False), N * ncm1).reshape(ncm1, N)
        assert (oracle.Oracle.canon(cm1).T == trace).all()
    finally:
        bufs.close()


def test_commit_witness_refuses_foreign_setup(dev):
    pkg, _ = dev
    lib = pkg.load()
    bogus = (ctypes.c_uint64 * 8)()
    setup = pkg.SetupC(ctypes.addressof(bogus), None)
    params = pkg.StepsParams()
    bufs = pkg.DeviceBuffers(arity=4)
    try:
        root = np.zeros(4, dtype=np.uint64)
        assert lib.commit_witness(ctypes.addressof(setup), ctypes.addressof(params), 0, 0, 0, root.ctypes.data,
                                  bufs.ptr, b"") == 2**64 - 1
        assert bufs.error() == pkg.B200_EINVAL
        assert b"StarkInfo" in lib.b200_last_error()
    finally:
        bufs.close()


def test_calculate_const_tree_from_starkinfo(dev, orc):
    """calculate_const_tree / get_const_tree_size on a stark_info_new pointer: nConstants columns."""
    pkg, _ = dev
    nbits, nbe, nconst = 11, 12, 6
    si = pkg.StarkInfo(write_setup(nbits, nbe, 3, 4, nconst))
    lib = pkg.load()
    size = int(lib.get_const_tree_size(si.ptr))
    assert size == (1 << nbe) * nconst + pkg.tree_num_elements(1 << nbe, 4)
    pols = oracle.random_field((1 << nbits, nconst), 77)
    out = np.zeros(size, dtype=np.uint64)
    lib.calculate_const_tree(si.ptr, pols.ctypes.data, out.ctypes.data, None)
    r_o, lde_o, tree_o = orc.commit(pols, nbe, 4)
    assert (out[:(1 << nbe) * nconst].reshape(nconst, 1 << nbe).T == lde_o).all()
    assert (out[(1 << nbe) * nconst:] == tree_o).all()
