"""CPU checkers for the commit path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may use this module, and only to check or time the CPU side.
The product (the CUDA library under ``pil2-proofman_b200/``) never imports it.

Two checkers, same interface (numpy uint64 arrays, canonical results):

* :class:`Oracle` — this project's plain-C restatement (``gl_oracle.c``).
* :class:`RefCPU` — the reference's own CPU sources (``NTT_Goldilocks``,
  ``Poseidon2Goldilocks<W>``) compiled unmodified into ``_ref/`` by the Makefile
  here.  The AVX-512 build is used where the host supports it, else AVX2.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = 0xFFFFFFFF00000001

_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_vp)


def reference_root():
    """The reference checkout: $PIL2_PROOFMAN_REF, else a directory `reference` beside this
    repository; None when neither holds pil2-stark (e.g. on a host that only runs prebuilt files)."""
    for cand in (os.environ.get("PIL2_PROOFMAN_REF"), os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                                   "reference")):
        if cand and os.path.isdir(os.path.join(cand, "pil2-stark")):
            return cand
    return None


def build(ref=True):
    """Compile the restatement (and, where the reference tree is present, _ref)."""
    targets = ["oracle"]
    extra = []
    root = reference_root()
    if ref and root:
        targets.append("ref")
        extra.append("REF=" + root)
    subprocess.run(["make", "-s", "-C", HERE] + targets + extra, check=True)


def tree_num_elements(nrows, arity):
    total, level = nrows, nrows
    while level > 1:
        total += (arity - level % arity) % arity
        level = (level + arity - 1) // arity
        total += level
    return total * 4


class _Base:
    lib = None

    def lde(self, trace, nbits_ext):
        """Row-major (N, ncols) -> row-major (NExt, ncols)."""
        trace = np.ascontiguousarray(trace, dtype=np.uint64)
        n, ncols = trace.shape
        out = np.zeros((1 << nbits_ext, ncols), dtype=np.uint64)
        self._lde(out, trace, n, 1 << nbits_ext, ncols)
        return self.canon(out)

    def merkletree(self, matrix, arity):
        """Row-major (nrows, ncols) -> full tree buffer (reference layout)."""
        matrix = np.ascontiguousarray(matrix, dtype=np.uint64)
        nrows, ncols = matrix.shape
        tree = np.zeros(tree_num_elements(nrows, arity), dtype=np.uint64)
        rc = self._merkletree(tree, matrix, ncols, nrows, arity)
        if rc != 0:
            raise ValueError("unsupported arity %d" % arity)
        return self.canon(tree)

    def commit(self, trace, nbits_ext, arity):
        """LDE + tree: returns (root[4], lde row-major, tree)."""
        lde = self.lde(trace, nbits_ext)
        tree = self.merkletree(lde, arity)
        return tree[-4:].copy(), lde, tree

    @staticmethod
    def canon(a):
        a = np.asarray(a, dtype=np.uint64)
        return np.where(a >= np.uint64(P), a - np.uint64(P), a)


class Oracle(_Base):
    """The C restatement in gl_oracle.c.  ``family`` selects the hash: 2 = Poseidon2 (default),
    1 = Poseidon1 (the reference's set_hash_family values)."""

    def __init__(self, family=2):
        self.family = 1 if family == 1 else 2
        path = os.path.join(HERE, "libgl_oracle.so")
        if not os.path.exists(path):
            build(ref=False)
        lib = ctypes.CDLL(path)
        for name, args in {
            "orc_lde": [_vp, _vp, _u64, _u64, _u64],
            "orc_ntt": [_vp, _vp, _u64, _u64, ctypes.c_int],
            "orc_merkletree": [_vp, _vp, _u64, _u64, _u64],
            "orc_merkletree_colmajor": [_vp, _vp, _u64, _u64, _u64],
            "orc_permute": [ctypes.c_uint, _vp],
            "orc_linear_hash": [ctypes.c_uint, _vp, _vp, _u64],
            "orc_merkletree_reduce": [ctypes.c_uint, _vp, _vp, _u64, _u64],
            "orc_tree_num_elements": [_u64, _u64],
            "orc_root_of_unity": [ctypes.c_uint],
            "orc_set_hash_family": [ctypes.c_int],
            "orc_group_proof": [_vp, _vp, _u64, _u64, _vp, _u64, _u64, _u64],
            "orc_root_from_proof": [_vp, _vp, _u64, _u64, _u64, _u64],
            "orc_commit_q": [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64],
            "orc_p1_permute": [ctypes.c_uint, _vp],
            "orc_merkletree_w": [ctypes.c_uint, _vp, _vp, _u64, _u64, _u64],
            "orc_mul": [_u64, _u64],
            "orc_add": [_u64, _u64],
            "orc_sub": [_u64, _u64],
        }.items():
            f = getattr(lib, name)
            f.argtypes = args
        for name in ("orc_tree_num_elements", "orc_root_of_unity", "orc_mul", "orc_add", "orc_sub",
                     "orc_group_proof"):
            getattr(lib, name).restype = _u64
        for name in ("orc_merkletree_w", "orc_merkletree", "orc_merkletree_colmajor", "orc_merkletree_reduce",
                     "orc_commit_q"):
            getattr(lib, name).restype = ctypes.c_int
        self.lib = lib

    def _lde(self, out, trace, n, next_, ncols):
        self.lib.orc_lde(_ptr(out), _ptr(trace), n, next_, ncols)

    def _fam(self):
        # the C library keeps the family in one global, like the reference's set_hash_family
        self.lib.orc_set_hash_family(self.family)

    def _merkletree(self, tree, matrix, ncols, nrows, arity):
        self._fam()
        return self.lib.orc_merkletree(_ptr(tree), _ptr(matrix), ncols, nrows, arity)

    def merkletree_w(self, width, matrix, arity):
        """Row-major matrix -> tree with sponge/node width `width` >= 4*arity (node input zero-padded)."""
        self._fam()
        matrix = np.ascontiguousarray(matrix, dtype=np.uint64)
        nrows, ncols = matrix.shape
        tree = np.zeros(tree_num_elements(nrows, arity), dtype=np.uint64)
        if self.lib.orc_merkletree_w(width, _ptr(tree), _ptr(matrix) if matrix.size else None, ncols, nrows,
                                     arity) != 0:
            raise ValueError("unsupported width/arity")
        return tree

    def merkletree_colmajor(self, cols, arity):
        """Column-major (ncols, nrows) -> tree."""
        cols = np.ascontiguousarray(cols, dtype=np.uint64)
        ncols, nrows = cols.shape
        tree = np.zeros(tree_num_elements(nrows, arity), dtype=np.uint64)
        self._fam()
        if self.lib.orc_merkletree_colmajor(_ptr(tree), _ptr(cols), ncols, nrows, arity) != 0:
            raise ValueError("unsupported arity")
        return tree

    def ntt(self, mat, inverse=False):
        mat = np.ascontiguousarray(mat, dtype=np.uint64)
        out = np.zeros_like(mat)
        self.lib.orc_ntt(_ptr(out), _ptr(mat), mat.shape[0], mat.shape[1], 1 if inverse else 0)
        return out

    def permute(self, state):
        st = np.ascontiguousarray(state, dtype=np.uint64).copy()
        if self.family == 1:
            self.lib.orc_p1_permute(len(st), _ptr(st))
        else:
            self.lib.orc_permute(len(st), _ptr(st))
        return st

    def linear_hash(self, width, data):
        self._fam()
        data = np.ascontiguousarray(data, dtype=np.uint64)
        out = np.zeros(4, dtype=np.uint64)
        self.lib.orc_linear_hash(width, _ptr(out), _ptr(data) if data.size else None, data.size)
        return out

    def merkletree_reduce(self, width, digests, arity):
        self._fam()
        digests = np.ascontiguousarray(digests, dtype=np.uint64)
        root = np.zeros(4, dtype=np.uint64)
        if self.lib.orc_merkletree_reduce(width, _ptr(root), _ptr(digests), digests.size // 4, arity) != 0:
            raise ValueError("width must be 4*arity")
        return root

    def group_proof(self, lde_rowmajor, tree, arity, row, llv=0):
        """MerkleTreeGL::getGroupProof of one row (row values + sibling digests)."""
        lde_rowmajor = np.ascontiguousarray(lde_rowmajor, dtype=np.uint64)
        tree = np.ascontiguousarray(tree, dtype=np.uint64)
        nrows, ncols = lde_rowmajor.shape
        out = np.zeros(ncols + 64 * 3 * 4, dtype=np.uint64)
        n = self.lib.orc_group_proof(_ptr(out), _ptr(lde_rowmajor), nrows, ncols, _ptr(tree), arity, llv, row)
        return out[:n].copy()

    def root_from_proof(self, proof, ncols, nrows, arity, row):
        proof = np.ascontiguousarray(proof, dtype=np.uint64)
        root = np.zeros(4, dtype=np.uint64)
        self._fam()
        self.lib.orc_root_from_proof(_ptr(root), _ptr(proof), ncols, nrows, arity, row)
        return root

    def commit_q(self, q, nbits, nbits_ext, qdeg, qdim, arity):
        """Starks::computeQ restated: q row-major (NExt, qDim) -> (root, cmQ row-major, tree)."""
        q = np.ascontiguousarray(q, dtype=np.uint64)
        next_ = 1 << nbits_ext
        root = np.zeros(4, dtype=np.uint64)
        cmq = np.zeros((next_, qdeg * qdim), dtype=np.uint64)
        tree = np.zeros(tree_num_elements(next_, arity), dtype=np.uint64)
        self._fam()
        if self.lib.orc_commit_q(_ptr(root), _ptr(cmq), _ptr(tree), _ptr(q), nbits, nbits_ext, qdeg, qdim, arity):
            raise ValueError("bad Q shape")
        return root, cmq, tree

    def root_of_unity(self, k):
        return int(self.lib.orc_root_of_unity(k))


def _cpu_has_avx512():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return " avx512f" in line
    except OSError:
        pass
    return False


class RefCPU(_Base):
    """The reference's CPU implementation, built unmodified into _ref/.  ``family`` 1 selects
    PoseidonGoldilocks<W> (Poseidon1), 2 Poseidon2Goldilocks<W>, as MerkleTreeGL::merkelize does."""

    def __init__(self, threads=None, family=2):
        self.family = 1 if family == 1 else 2
        variant = "avx512" if _cpu_has_avx512() else "avx2"
        path = os.path.join(HERE, "_ref", "libpil2ref_%s.so" % variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with: make -C oracle ref)")
        lib = ctypes.CDLL(path)
        lib.ref_lde.argtypes = [_vp, _vp, _u64, _u64, _u64, _vp, _u64]
        lib.ref_ntt.argtypes = [_vp, _vp, _u64, _u64, ctypes.c_int]
        lib.ref_merkletree.argtypes = [_vp, _vp, _u64, _u64, _u64]
        lib.ref_merkletree.restype = ctypes.c_int
        lib.ref_permute.argtypes = [_u64, _vp, _vp]
        lib.ref_linear_hash.argtypes = [_u64, _vp, _vp, _u64]
        lib.ref_merkletree_reduce.argtypes = [_u64, _vp, _vp, _u64, _u64]
        lib.ref_tree_num_elements.argtypes = [_u64, _u64]
        lib.ref_tree_num_elements.restype = _u64
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_max_threads.restype = ctypes.c_int
        lib.ref_canonicalize.argtypes = [_vp, _u64]
        lib.ref_p1_permute.argtypes = [_u64, _vp, _vp]
        lib.ref_p1_linear_hash.argtypes = [_u64, _vp, _vp, _u64]
        lib.ref_p1_merkletree.argtypes = [_u64, _vp, _vp, _u64, _u64, _u64]
        lib.ref_p1_merkletree.restype = ctypes.c_int
        lib.ref_commit_q.argtypes = [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64]
        lib.ref_commit_q.restype = ctypes.c_int
        lib.ref_fill_random.argtypes = [_vp, _u64, _u64]
        self.lib = lib
        self.variant = variant
        if threads:
            lib.ref_set_threads(int(threads))

    @property
    def threads(self):
        return int(self.lib.ref_max_threads())

    def _lde(self, out, trace, n, next_, ncols):
        self.lib.ref_lde(_ptr(out), _ptr(trace), n, next_, ncols, None, 1)

    def _merkletree(self, tree, matrix, ncols, nrows, arity):
        if self.family == 1:
            return self.lib.ref_p1_merkletree(0, _ptr(tree), _ptr(matrix), ncols, nrows, arity)
        return self.lib.ref_merkletree(_ptr(tree), _ptr(matrix), ncols, nrows, arity)

    def merkletree_w(self, width, matrix, arity):
        """Poseidon1 merkletree<width> with 4*arity <= width (row-major matrix)."""
        matrix = np.ascontiguousarray(matrix, dtype=np.uint64)
        nrows, ncols = matrix.shape
        tree = np.zeros(tree_num_elements(nrows, arity), dtype=np.uint64)
        if self.family != 1 or self.lib.ref_p1_merkletree(width, _ptr(tree), _ptr(matrix) if matrix.size else None,
                                                          ncols, nrows, arity) != 0:
            raise ValueError("unsupported width/arity")
        return self.canon(tree)

    def permute(self, state):
        st = np.ascontiguousarray(state, dtype=np.uint64)
        out = np.zeros_like(st)
        (self.lib.ref_p1_permute if self.family == 1 else self.lib.ref_permute)(len(st), _ptr(out), _ptr(st))
        return self.canon(out)

    def linear_hash(self, width, data):
        data = np.ascontiguousarray(data, dtype=np.uint64)
        out = np.zeros(4, dtype=np.uint64)
        f = self.lib.ref_p1_linear_hash if self.family == 1 else self.lib.ref_linear_hash
        f(width, _ptr(out), _ptr(data) if data.size else None, data.size)
        return self.canon(out)

    def merkletree_reduce(self, width, digests, arity):
        digests = np.ascontiguousarray(digests, dtype=np.uint64)
        root = np.zeros(4, dtype=np.uint64)
        self.lib.ref_merkletree_reduce(width, _ptr(root), _ptr(digests), digests.size // 4, arity)
        return self.canon(root)

    def ntt(self, mat, inverse=False):
        mat = np.ascontiguousarray(mat, dtype=np.uint64)
        out = np.zeros_like(mat)
        self.lib.ref_ntt(_ptr(out), _ptr(mat), mat.shape[0], mat.shape[1], 1 if inverse else 0)
        return self.canon(out)

    def lde_raw(self, trace, nbits_ext, out=None, buffer=None, nblock=1):
        """Uncanonicalised LDE into a caller buffer (timing path).  ``buffer`` (optional) is the
        NTT's work area of NExt x ceil(ncols / nblock) words; without it the reference allocates
        NExt x ncols words itself."""
        n, ncols = trace.shape
        if out is None:
            out = np.empty((1 << nbits_ext, ncols), dtype=np.uint64)
        if buffer is not None:
            assert buffer.size >= (1 << nbits_ext) * -(-ncols // nblock)
        self.lib.ref_lde(_ptr(out), _ptr(trace), n, 1 << nbits_ext, ncols, _ptr(buffer),
                         nblock if buffer is not None else 1)
        return out

    def commit_q(self, q, nbits, nbits_ext, qdeg, qdim, arity):
        """Starks::computeQ on the reference's NTT: q row-major (NExt, qDim) -> (root, cmQ
        row-major (NExt, qDeg*qDim), tree), all canonical."""
        q = np.ascontiguousarray(q, dtype=np.uint64)
        next_ = 1 << nbits_ext
        root = np.zeros(4, dtype=np.uint64)
        cmq = np.zeros((next_, qdeg * qdim), dtype=np.uint64)
        tree = np.zeros(tree_num_elements(next_, arity), dtype=np.uint64)
        if self.lib.ref_commit_q(_ptr(root), _ptr(cmq), _ptr(tree), _ptr(q), nbits, nbits_ext, qdeg, qdim, arity):
            raise ValueError("bad Q shape")
        return self.canon(root), self.canon(cmq), self.canon(tree)

    def fill_random(self, n, seed):
        """n seeded field elements, the same rule as the product's fill_random (splitmix64 keyed by
        (seed, index), rejection below p), filled with every OpenMP thread."""
        out = np.empty(n, dtype=np.uint64)
        self.lib.ref_fill_random(_ptr(out), n, seed)
        return out

    def merkletree_raw(self, matrix, arity, tree=None):
        """Uncanonicalised tree of a row-major matrix into a caller buffer (timing path), with the
        family this checker was created for."""
        nrows, ncols = matrix.shape
        if tree is None:
            tree = np.empty(tree_num_elements(nrows, arity), dtype=np.uint64)
        if self.family == 1:
            self.lib.ref_p1_merkletree(0, _ptr(tree), _ptr(matrix), ncols, nrows, arity)
        else:
            self.lib.ref_merkletree(_ptr(tree), _ptr(matrix), ncols, nrows, arity)
        return tree


def random_field(shape, seed):
    """Uniform elements of [0, p) from a seeded PCG64 stream, by rejection."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = int(np.prod(shape))
    out = np.empty(n, dtype=np.uint64)
    filled = 0
    while filled < n:
        draw = rng.integers(0, 2**64, size=n - filled, dtype=np.uint64, endpoint=False)
        draw = draw[draw < np.uint64(P)]
        out[filled:filled + draw.size] = draw
        filled += draw.size
    return out.reshape(shape)
