"""Python host mirror of the pil2_b200 C ABI (include/pil2_b200.h).

The product is the CUDA shared library ``libpil2_b200.so`` built from ``csrc/`` for
sm_100a; this module only binds it with ctypes, mirroring the reference's commit
entry points (pil2-stark/src/api/starks_api.hpp) and the native ``b200_*`` API.
There is no CPU fallback: if the library is missing or no GPU is present, calls fail.

Device buffers are passed as raw pointers; torch tensors (dtype int64 or uint64,
used only as 64-bit storage) are accepted wherever a device pointer is expected.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpil2_b200.so")
P = 0xFFFFFFFF00000001

B200_OK = 0
B200_EINVAL = -1
B200_ECUDA = -2
B200_ENOMEM = -3
B200_EFAMILY = -4
B200_EBUSY = -5
B200_ETIMEOUT = -6

_u64 = ctypes.c_uint64
_i32 = ctypes.c_int
_vp = ctypes.c_void_p
_pu64 = ctypes.POINTER(ctypes.c_uint64)

_SIGS = {
    # reference ABI
    "set_hash_family": (None, [ctypes.c_uint8]),
    "init_gpu_setup": (None, [_u64]),
    "gen_device_buffers": (_vp, [ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_uint32, ctypes.c_uint32]),
    "free_device_buffers": (None, [_vp]),
    "gen_device_streams": (_u64, [_vp, _u64, _u64, _vp, _u64, _u64, _u64]),
    "write_custom_commit": (None, [_vp, _u64, _u64, _u64, _u64, _vp, _vp, ctypes.c_char_p]),
    "commit_witness": (_u64, [_vp, _vp, _u64, _u64, _u64, _vp, _vp, ctypes.c_char_p]),
    "get_stream_proofs": (None, [_vp]),
    "get_stream_proofs_non_blocking": (None, [_vp]),
    "wait_trace_h2d_done": (None, [_vp, _u64]),
    "calculate_const_tree": (None, [_vp, _vp, _vp, _vp]),
    "get_const_tree_size": (_u64, [_vp]),
    "set_gpu_mode": (ctypes.c_bool, [ctypes.c_bool]),
    "stark_info_new": (_vp, [ctypes.c_char_p] + [ctypes.c_bool] * 7),
    "stark_info_free": (None, [_vp]),
    "get_map_total_n": (_u64, [_vp]),
    "get_map_total_n_custom_commits_fixed": (_u64, [_vp]),
    "get_map_total_n_contributions": (_u64, [_vp]),
    "get_const_size": (_u64, [_vp]),
    # native
    "b200_stark_shape_new": (_vp, [_u64, _u64, _u64, _u64]),
    "b200_stark_shape_free": (None, [_vp]),
    "b200_stark_info_offset": (_u64, [_vp, ctypes.c_char_p, _i32]),
    "b200_stark_info_value": (_u64, [_vp, ctypes.c_char_p]),
    "b200_commit_buffers_aux": (_i32, [_vp, _u64, ctypes.POINTER(_vp), _pu64]),
    "b200_last_error": (ctypes.c_char_p, []),
    "b200_buffers_error": (_i32, [_vp]),
    "b200_init": (_i32, [_i32]),
    "b200_device_count": (_i32, []),
    "b200_tree_num_elements": (_u64, [_u64, _u64]),
    "b200_set_native_hash_family": (_i32, [_i32]),
    "b200_native_hash_family": (_i32, []),
    "b200_lde_scratch_words": (_u64, [_u64, _u64]),
    "b200_lde_device": (_i32, [_vp, _vp, _i32, _u64, _u64, _u64, _vp, _vp]),
    "b200_lde_device_static_scratch": (_i32, [_vp, _vp, _i32, _u64, _u64, _u64, _vp]),
    "b200_merkletree_device": (_i32, [_vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "b200_commit_device": (_i32, [_vp, _vp, _vp, _vp, _i32, _u64, _u64, _u64, _u64, _vp, _vp]),
    "b200_permute_device": (_i32, [_vp, _vp, _u64, _u64, _vp]),
    "b200_commit_host": (_i32, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64]),
    "b200_fill_random_device": (_i32, [_vp, _u64, _u64, _vp]),
    "b200_fill_random_host": (None, [_vp, _u64, _u64]),
    "b200_lde_rows_device": (_i32, [_vp, _vp, _u64, _u64, _vp, _u64, _vp]),
    "register_host_memory": (ctypes.c_uint32, [_vp, _u64]),
    "unregister_host_memory": (None, [_vp]),
    "b200_kernel_names": (ctypes.c_char_p, []),
    "b200_timing_enable": (None, [_i32]),
    "b200_timing_reset": (None, []),
    "b200_timing_get": (_i32, [_i32, ctypes.POINTER(ctypes.c_double), _pu64]),
    "b200_timing_name": (ctypes.c_char_p, [_i32]),
    "b200_launch_count": (_u64, []),
    "b200_set_transpose_tma": (_i32, [_i32]),
    "b200_tma_wait_errors": (_i32, []),
    "b200_probe_imad": (_i32, [_u64, _u64, ctypes.POINTER(ctypes.c_double)]),
    "b200_batch_plan_new": (_vp, [_vp, _u64]),
    "b200_batch_plan_run": (_i32, [_vp, _vp, _vp, _i32]),
    "b200_batch_plan_free": (None, [_vp]),
    "b200_batch_plan_launches": (_u64, [_vp]),
    "b200_commit_batch_device": (_i32, [_vp, _u64, _vp, _vp]),
    "b200_server_new": (_vp, [_i32, _u64, ctypes.c_uint32]),
    "b200_server_submit": (ctypes.c_int64, [_vp, _vp, _u64, _u64, _u64, _u64, _vp]),
    "b200_server_status": (_i32, [_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]),
    "b200_server_wait_all": (_i32, [_vp, _u64]),
    "b200_server_release": (_i32, [_vp, ctypes.c_int64]),
    "b200_server_buffers": (_i32, [_vp, ctypes.c_int64, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
    "b200_server_free": (None, [_vp]),
    "b200_server_configure": (_i32, [_vp, _i32, _u64, ctypes.c_uint32]),
    "b200_server_stats": (_i32, [_vp, _pu64, _u64]),
    "b200_server_request_times": (_i32, [_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]),
    "b200_server_request_gpu_times": (_i32, [_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]),
    # query openings, Q stage, plan autotuner, packed witness
    "b200_query_proof_words": (_u64, [_u64, _u64, _u64, _u64]),
    "b200_query_openings_device": (_i32, [_vp, _vp, _u64, _u64, _vp, _u64, _u64, _vp, _u64, _vp]),
    "b200_q_scratch_words": (_u64, [_u64, _u64]),
    "b200_commit_q_device": (_i32, [_vp, _vp, _vp, _vp, _i32, _u64, _u64, _u64, _u64, _u64, _vp, _vp]),
    "b200_autotune_lde": (_i32, [_u64, _u64, _u64, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "b200_autotune_get": (None, [_u64, _u64, _u64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "b200_autotune_set": (None, [_u64, _u64, _u64, ctypes.c_uint32, ctypes.c_uint32]),
    "b200_autotune_save": (_i32, [ctypes.c_char_p]),
    "b200_autotune_load": (_i32, [ctypes.c_char_p]),
    "b200_packed_words_per_row": (_u64, [_vp, _u64]),
    "b200_commit_packed_device": (_i32, [_vp, _vp, _vp, _vp, _u64, _vp, _u64, _u64, _u64, _u64, _vp, _vp]),
    # streaming slot commit
    "stream_commit_slot_bytes": (_u64, [_u64, _u64, _u64, _u64]),
    "configure_stream_commit_slots": (None, [_vp, _u64, _u64]),
    "get_stream_commit_slots": (_u64, [_vp]),
    "get_stream_commit_floor": (_u64, [_vp]),
    "commit_witness_streaming": (ctypes.c_int64, [_vp, _u64, _u64, _u64, _vp, _u64, _u64, _u64, _u64, _vp, _vp]),
    "stream_commit_pause": (None, []),
    "b200_stream_commit_packed": (_i32, [_vp, _u64, _vp, _u64, _u64, _u64, _u64, _vp, _vp, _vp]),
    "b200_tree_last_level_words": (_u64, [_u64, _u64]),
    "b200_tree_last_level_device": (_i32, [_vp, _vp, _u64, _u64, _u64, _vp]),
    "b200_merkletree_reduce_device": (_i32, [_vp, _vp, _u64, _u64, _vp, _vp]),
    # indexed witness
    "register_instruction_table": (None, [_vp, _u64, _u64, _vp, _u64, _u64]),
    "b200_register_indexed_air": (_i32, [_vp, _u64, _u64, _u64, _vp, _u64]),
    "b200_commit_indexed_device": (_i32, [_vp, _vp, _vp, _vp, _u64, _vp, _u64, _u64, _u64, _vp, _vp, _u64, _u64,
                                          _u64, _u64, _vp, _vp]),
    "b200_stream_commit_indexed": (_i32, [_vp, _u64, _vp, _u64, _u64, _u64, _u64, _vp, _vp, _u64, _vp, _u64, _u64,
                                          _vp, _vp]),
}

_lib = None


def load(path=LIB_PATH):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("%s is missing: build it with `python %s`" % (path, os.path.join(HERE, "build.py")))
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(_SIGS)


class B200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("pil2_b200 error %d: %s" % (code, msg))
        self.code = code


def _check(rc):
    if rc != 0:
        raise B200Error(rc, (load().b200_last_error() or b"").decode())
    return rc


def _ptr(x):
    """Device/host pointer of a torch tensor, numpy array, int or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        assert x.dtype == np.uint64 and x.flags["C_CONTIGUOUS"]
        return x.ctypes.data
    # torch tensor
    assert x.element_size() == 8 and x.is_contiguous()
    return x.data_ptr()


def _stream(stream):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream  # torch.cuda.Stream


def tree_num_elements(nrows, arity):
    return int(load().b200_tree_num_elements(nrows, arity))


def lde_scratch_words(nbits, ncols):
    return int(load().b200_lde_scratch_words(nbits, ncols))


def init(device=0):
    _check(load().b200_init(device))


# ---------------------------------------------------------------- native API ----

def lde_device(d_lde, d_trace, nbits, nbits_ext, ncols, d_scratch, trace_rowmajor=True, stream=None):
    _check(load().b200_lde_device(_ptr(d_lde), _ptr(d_trace), 1 if trace_rowmajor else 0, nbits, nbits_ext,
                                  ncols, _ptr(d_scratch), _stream(stream)))


def lde_device_static_scratch(d_lde, d_trace, nbits, nbits_ext, ncols, trace_rowmajor=True, stream=None):
    """LDE without any device allocation: the scratch is the library's built-in 64 MiB array
    (N * nCols <= 2^23).  Calls share that array, so calls that overlap on the GPU race."""
    _check(load().b200_lde_device_static_scratch(_ptr(d_lde), _ptr(d_trace), 1 if trace_rowmajor else 0, nbits,
                                                 nbits_ext, ncols, _stream(stream)))


def merkletree_device(d_tree, d_src, rs, cs, ncols, nrows, arity, stream=None):
    _check(load().b200_merkletree_device(_ptr(d_tree), _ptr(d_src), rs, cs, ncols, nrows, arity, _stream(stream)))


def commit_device(d_lde, d_tree, d_trace, nbits, nbits_ext, ncols, arity, d_scratch, trace_rowmajor=True,
                  stream=None, want_root=True):
    root = np.zeros(4, dtype=np.uint64) if want_root else None
    _check(load().b200_commit_device(_ptr(root), _ptr(d_lde), _ptr(d_tree), _ptr(d_trace),
                                     1 if trace_rowmajor else 0, nbits, nbits_ext, ncols, arity, _ptr(d_scratch),
                                     _stream(stream)))
    return root


def permute_device(d_out, d_in, n, width, stream=None):
    _check(load().b200_permute_device(_ptr(d_out), _ptr(d_in), n, width, _stream(stream)))


def fill_random_device(d_buf, n, seed, stream=None):
    _check(load().b200_fill_random_device(_ptr(d_buf), n, seed, _stream(stream)))


def fill_random_host(n, seed):
    out = np.empty(n, dtype=np.uint64)
    load().b200_fill_random_host(_ptr(out), n, seed)
    return out


def lde_rows_device(d_out, d_lde, next_, ncols, d_rows, nreq, stream=None):
    _check(load().b200_lde_rows_device(_ptr(d_out), _ptr(d_lde), next_, ncols, _ptr(d_rows), nreq, _stream(stream)))


def commit_host(trace, nbits_ext, arity, want_lde=False, want_tree=False):
    """Row-major (N, nCols) uint64 trace -> (root[4], lde column-major (nCols, NExt) or None, tree or None)."""
    trace = np.ascontiguousarray(trace, dtype=np.uint64)
    n, ncols = trace.shape
    nbits = n.bit_length() - 1
    assert 1 << nbits == n
    next_ = 1 << nbits_ext
    root = np.zeros(4, dtype=np.uint64)
    lde = np.zeros((ncols, next_), dtype=np.uint64) if want_lde else None
    tree = np.zeros(tree_num_elements(next_, arity), dtype=np.uint64) if want_tree else None
    _check(load().b200_commit_host(_ptr(root), _ptr(lde), _ptr(tree), _ptr(trace), nbits, nbits_ext, ncols, arity))
    return root, lde, tree


def kernel_names():
    return load().b200_kernel_names().decode().split()


# ------------------------------------------------------------ reference ABI ----

class StepsParams(ctypes.Structure):
    """starkpil/steps.hpp:6-20 — twelve pointers; commit_witness reads `trace`."""
    _fields_ = [(n, ctypes.c_void_p) for n in (
        "trace", "aux_trace", "publicInputs", "proofValues", "challenges", "airgroupValues", "airValues",
        "evals", "xDivXSub", "pConstPolsAddress", "pConstPolsExtendedTreeAddress", "pCustomCommitsFixed")]


class BatchInstance(ctypes.Structure):
    """B200BatchInstance: device buffers and shape of one instance of a batched commit."""
    _fields_ = [("d_trace", ctypes.c_void_p), ("d_scratch", ctypes.c_void_p), ("d_lde", ctypes.c_void_p),
                ("d_tree", ctypes.c_void_p), ("nBits", ctypes.c_uint64), ("nBitsExt", ctypes.c_uint64),
                ("nCols", ctypes.c_uint64), ("arity", ctypes.c_uint64)]


class SetupC(ctypes.Structure):
    """proofman's SetupC (common/src/setup.rs:45-57): what commit_witness receives as pSetupCtx."""
    _fields_ = [("p_stark_info", ctypes.c_void_p), ("p_expressions_bin", ctypes.c_void_p)]


class StarkInfo:
    """Owns a StarkInfo of the library: from a starkinfo JSON file (stark_info_new, starks_api.hpp:37)
    or, with from_shape, from the commit's four numbers.  ``ptr`` is the pStarkInfo of
    calculate_const_tree / get_const_tree_size; ``setup_ptr`` points to a SetupC holding it, the
    pSetupCtx of commit_witness."""

    def __init__(self, path=None, recursive_final=False, recursive=False, verify_constraints=False, verify=False,
                 gpu=True, preallocate=False, single_use=False, _ptr=None):
        lib = load()
        if _ptr is None:
            _ptr = lib.stark_info_new(os.fsencode(path), recursive_final, recursive, verify_constraints, verify, gpu,
                                      preallocate, single_use)
            if not _ptr:
                raise B200Error(B200_EINVAL, (lib.b200_last_error() or b"").decode())
        self.ptr = _ptr
        self.setup = SetupC(self.ptr, None)
        self.setup_ptr = ctypes.addressof(self.setup)

    @classmethod
    def from_shape(cls, nbits, nbits_ext, ncols, arity):
        return cls(_ptr=load().b200_stark_shape_new(nbits, nbits_ext, ncols, arity))

    def offset(self, section, extended):
        v = int(load().b200_stark_info_offset(self.ptr, section.encode(), 1 if extended else 0))
        return None if v == 2**64 - 1 else v

    def value(self, name):
        v = int(load().b200_stark_info_value(self.ptr, name.encode()))
        return None if v == 2**64 - 1 else v

    def map_total_n(self):
        return int(load().get_map_total_n(self.ptr))

    def map_total_n_contributions(self):
        return int(load().get_map_total_n_contributions(self.ptr))

    def close(self):
        if getattr(self, "ptr", None) and _lib is not None:
            _lib.stark_info_free(self.ptr)
        self.ptr = None

    def __del__(self):
        self.close()


class StarkShape(StarkInfo):
    """A StarkInfo from the commit's four numbers (b200_stark_shape_new)."""

    def __init__(self, nbits, nbits_ext, ncols, arity):
        super().__init__(_ptr=load().b200_stark_shape_new(nbits, nbits_ext, ncols, arity))
        self.nbits, self.nbits_ext, self.ncols, self.arity = nbits, nbits_ext, ncols, arity


class DeviceBuffers:
    """gen_device_buffers / free_device_buffers (starks_api.hpp:190,193)."""

    def __init__(self, arity=4, max_n_bits_ext=0, n_streams=2):
        lib = load()
        self.ptr = lib.gen_device_buffers(0, 1, None, arity, max_n_bits_ext)
        if not self.ptr:
            raise B200Error(B200_ENOMEM, (lib.b200_last_error() or b"").decode())
        if n_streams != 2:
            lib.gen_device_streams(self.ptr, n_streams, 0, None, 0, 0, arity)

    def error(self):
        return int(load().b200_buffers_error(self.ptr))

    def aux(self, stream_id):
        """(device pointer, words) of stream slot stream_id's prover buffer (after its harvest)."""
        p, n = ctypes.c_void_p(), ctypes.c_uint64()
        _check(load().b200_commit_buffers_aux(self.ptr, stream_id, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def close(self):
        if self.ptr:
            load().free_device_buffers(self.ptr)
            self.ptr = None

    def __del__(self):
        if _lib is not None:
            self.close()


def set_hash_family(fam):
    load().set_hash_family(fam)


# ----------------------------------------------------------------- profiling ----

TIMING_CATEGORIES = ("transpose", "ntt_inverse", "ntt_forward", "leaf_hash", "tree_levels")


def timing_enable(on=True):
    load().b200_timing_enable(1 if on else 0)


def timing_reset():
    load().b200_timing_reset()


def timing():
    """{category: (total_ms, launch_groups)} since the last reset (waits for the events)."""
    lib = load()
    out = {}
    for i, name in enumerate(TIMING_CATEGORIES):
        ms = ctypes.c_double()
        cnt = ctypes.c_uint64()
        _check(lib.b200_timing_get(i, ctypes.byref(ms), ctypes.byref(cnt)))
        out[name] = (ms.value, cnt.value)
    return out


def launch_count():
    return int(load().b200_launch_count())


def probe_imad(blocks=148 * 16, iters=1 << 16):
    r = ctypes.c_double()
    _check(load().b200_probe_imad(blocks, iters, ctypes.byref(r)))
    return r.value



# ---------------------------------------------------------------- query openings ----
def query_proof_words(next_, ncols, arity, llv=0):
    """Words of one opening (MerkleTreeGL::getGroupProof layout)."""
    return int(load().b200_query_proof_words(next_, ncols, arity, llv))


def query_openings_device(d_out, d_lde, next_, ncols, d_tree, arity, d_rows, nqueries, llv=0, stream=None):
    _check(load().b200_query_openings_device(_ptr(d_out), _ptr(d_lde), next_, ncols, _ptr(d_tree), arity, llv,
                                             _ptr(d_rows), nqueries, _stream(stream)))


# ---------------------------------------------------------------- Q stage ----
def q_scratch_words(nbits_ext, qdim):
    return int(load().b200_q_scratch_words(nbits_ext, qdim))


def commit_q_device(d_cmq, d_tree, d_q, nbits, nbits_ext, qdeg, qdim, arity, d_scratch, q_rowmajor=True,
                    stream=None):
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_commit_q_device(_ptr(root), _ptr(d_cmq), _ptr(d_tree), _ptr(d_q), 1 if q_rowmajor else 0,
                                       nbits, nbits_ext, qdeg, qdim, arity, _ptr(d_scratch), _stream(stream)))
    return root


# ---------------------------------------------------------------- plan autotuner ----
def autotune_lde(nbits, nbits_ext, ncols):
    """Time every window plan for this shape; returns (best ms on the probe, kfirst, krest)."""
    ms, kf, kr = ctypes.c_double(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(load().b200_autotune_lde(nbits, nbits_ext, ncols, ctypes.byref(ms), ctypes.byref(kf), ctypes.byref(kr)))
    return ms.value, kf.value, kr.value


def autotune_get(nbits, nbits_ext, ncols):
    kf, kr = ctypes.c_uint32(), ctypes.c_uint32()
    load().b200_autotune_get(nbits, nbits_ext, ncols, ctypes.byref(kf), ctypes.byref(kr))
    return kf.value, kr.value


def autotune_set(nbits, nbits_ext, ncols, kfirst, krest):
    load().b200_autotune_set(nbits, nbits_ext, ncols, kfirst, krest)


def autotune_save(path):
    _check(load().b200_autotune_save(path.encode()))


def autotune_load(path):
    _check(load().b200_autotune_load(path.encode()))


# ---------------------------------------------------------------- packed witness ----
def packed_words_per_row(col_bits):
    bits = np.ascontiguousarray(col_bits, dtype=np.uint32)
    return int(load().b200_packed_words_per_row(bits.ctypes.data, bits.size))


def commit_packed_device(d_lde, d_tree, d_packed, words_per_row, col_bits, nbits, nbits_ext, arity, d_scratch,
                         stream=None):
    bits = np.ascontiguousarray(col_bits, dtype=np.uint32)
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_commit_packed_device(_ptr(root), _ptr(d_lde), _ptr(d_tree), _ptr(d_packed), words_per_row,
                                            bits.ctypes.data if bits.size else None, nbits, nbits_ext, bits.size,
                                            arity, _ptr(d_scratch), _stream(stream)))
    return root


def pack_rows(trace, col_bits):
    """Host packer (row-major trace, per-column widths) -> (N, words_per_row) uint64: the inverse of the
    device unpack, used by tests and benchmarks to build packed witnesses."""
    trace = np.ascontiguousarray(trace, dtype=np.uint64)
    n, ncols = trace.shape
    bits = [int(b) for b in col_bits]
    wpr = (sum(bits) + 63) // 64
    out = np.zeros((n, wpr), dtype=np.uint64)
    off = 0
    for c, nb in enumerate(bits):
        mask = np.uint64((1 << nb) - 1) if nb < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
        v = trace[:, c] & mask
        w, o = divmod(off, 64)
        out[:, w] |= v << np.uint64(o)
        if o + nb > 64:
            out[:, w + 1] |= v >> np.uint64(64 - o)
        off += nb
    return out


# ---------------------------------------------------------------- hash family ----
def set_native_hash_family(family):
    """1 = Poseidon1, 2 = Poseidon2 (default) for the native b200_* entry points."""
    _check(load().b200_set_native_hash_family(family))


def native_hash_family():
    return int(load().b200_native_hash_family())


# ---------------------------------------------------------------- streaming slot commit ----
def stream_commit_slot_bytes(nbits, nbits_ext, ncols, words_per_row):
    return int(load().stream_commit_slot_bytes(nbits, nbits_ext, ncols, words_per_row))


def stream_commit_packed(d_slot, slot_words, packed, col_bits, nbits, nbits_ext, stream=None):
    """Native streaming commit of host packed rows (N, words_per_row); returns the root."""
    packed = np.ascontiguousarray(packed, dtype=np.uint64)
    widths = np.ascontiguousarray(col_bits, dtype=np.uint64)
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_stream_commit_packed(_ptr(d_slot), slot_words, packed.ctypes.data, nbits, nbits_ext,
                                            widths.size, packed.shape[1], widths.ctypes.data, root.ctypes.data,
                                            _stream(stream)))
    return root


# ---------------------------------------------------------------- indexed witness ----
def pack_indexed(runtime, index, index_bits, table_vals, col_bits, col_source):
    """Host packer of an indexed witness.  runtime: (N, nRuntime) values of the source-0 columns in
    column order; index: (N,) entry per row; table_vals: (E, nTable) values of the source-1 columns.
    Returns (rows (N, words_per_row), table (E, words_per_entry))."""
    col_bits = [int(b) for b in col_bits]
    src = [int(x) for x in col_source]
    rt_bits = [b for b, x in zip(col_bits, src) if not x]
    tb_bits = [b for b, x in zip(col_bits, src) if x]
    runtime = np.ascontiguousarray(runtime, dtype=np.uint64).reshape(len(index), len(rt_bits))
    parts, widths = [], []
    if index_bits:
        parts.append(np.asarray(index, dtype=np.uint64)[:, None])
        widths.append(index_bits)
    parts.append(runtime)
    widths += rt_bits
    rows = pack_rows(np.concatenate(parts, axis=1), widths) if widths else np.zeros((len(index), 1), np.uint64)
    table_vals = np.ascontiguousarray(table_vals, dtype=np.uint64)
    if not tb_bits:
        return rows, np.zeros((max(1, table_vals.shape[0] if table_vals.ndim else 1), 0), np.uint64)
    table = pack_rows(table_vals.reshape(-1, len(tb_bits)), tb_bits)
    return rows, table


def commit_indexed_device(d_lde, d_tree, d_rows, words_per_row, d_table, num_entries, words_per_entry, index_bits,
                          col_bits, col_source, nbits, nbits_ext, arity, d_scratch, stream=None):
    bits = np.ascontiguousarray(col_bits, dtype=np.uint64)
    srcs = np.ascontiguousarray(col_source, dtype=np.uint8)
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_commit_indexed_device(_ptr(root), _ptr(d_lde), _ptr(d_tree), _ptr(d_rows), words_per_row,
                                             _ptr(d_table), num_entries, words_per_entry, index_bits,
                                             bits.ctypes.data, srcs.ctypes.data, nbits, nbits_ext, bits.size, arity,
                                             _ptr(d_scratch), _stream(stream)))
    return root


def stream_commit_indexed(d_slot, slot_words, rows, col_bits, col_source, index_bits, d_table, num_entries,
                          words_per_entry, nbits, nbits_ext, stream=None):
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    bits = np.ascontiguousarray(col_bits, dtype=np.uint64)
    srcs = np.ascontiguousarray(col_source, dtype=np.uint8)
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_stream_commit_indexed(_ptr(d_slot), slot_words, rows.ctypes.data, nbits, nbits_ext, bits.size,
                                             rows.shape[1], bits.ctypes.data, srcs.ctypes.data, index_bits,
                                             _ptr(d_table), num_entries, words_per_entry, root.ctypes.data,
                                             _stream(stream)))
    return root


# ---------------------------------------------------------------- tree level, digest reduction ----
def tree_last_level_device(d_out, d_tree, next_, arity, llv, stream=None):
    _check(load().b200_tree_last_level_device(_ptr(d_out), _ptr(d_tree), next_, arity, llv, _stream(stream)))


def merkletree_reduce_device(d_digests, n, arity, d_tree, stream=None):
    root = np.zeros(4, dtype=np.uint64)
    _check(load().b200_merkletree_reduce_device(root.ctypes.data, _ptr(d_digests), n, arity, _ptr(d_tree),
                                                _stream(stream)))
    return root
