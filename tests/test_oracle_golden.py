"""Pin the CPU oracle (and the compiled reference CPU path) to the reference's known answers.

Sources of the vectors: tests/golden/reference_kats.json, written by make_golden.py from
the reference test sources (goldilocks/tests/test_helpers.hpp:17-66,
test_ntt_cpu.cpp:182-412) and from the reference CPU build on seeded inputs.
"""
import hashlib

import numpy as np
import pytest

import oracle

P = oracle.P


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


@pytest.mark.parametrize("w", [4, 8, 12, 16])
def test_permute_golden(orc, kats, w):
    out = orc.permute(np.arange(w, dtype=np.uint64))
    assert [int(v) for v in out] == kats["poseidon2"]["PERMUTE_W%d_GOLDEN" % w]
    assert [int(v) for v in out[:4]] == kats["poseidon2"]["PERMUTE_TRUNC_W%d_GOLDEN" % w]


@pytest.mark.parametrize("w", [8, 12, 16])
def test_linear_hash_golden(orc, kats, w):
    out = orc.linear_hash(w, np.arange(1, 21, dtype=np.uint64))
    assert [int(v) for v in out] == kats["poseidon2"]["LINEAR_HASH_W%d_GOLDEN" % w]


def test_linear_hash_empty_is_zero(orc):
    # size 0 -> zero digest (test_poseidon2_cpu.cpp:375-389)
    assert orc.linear_hash(16, np.zeros(0, dtype=np.uint64)).tolist() == [0, 0, 0, 0]


def test_merkletree_reduce_golden(orc, kats):
    root = orc.merkletree_reduce(12, np.arange(1, 13, dtype=np.uint64), 3)
    assert [int(v) for v in root] == kats["poseidon2"]["MERKLETREE_REDUCE_W12_AR3_GOLDEN"]


def _pmul(a, b):
    return (a * b) % P


def test_lde_block_golden(orc, kats):
    # 8 columns, rows 0,1 = 1 + col, then Fibonacci; N=16 -> 32 (test_ntt_cpu.cpp:264-350)
    n, ncols = 16, 8
    a = [[0] * ncols for _ in range(n)]
    for j in range(ncols):
        a[0][j] = a[1][j] = 1 + j
    for i in range(2, n):
        for j in range(ncols):
            a[i][j] = (a[i - 1][j] + a[i - 2][j]) % P
    lde = orc.lde(np.array(a, dtype=np.uint64), 5)
    assert [int(v) for v in lde[:, 0]] == kats["lde_block_16_32_col0"]


def test_lde_explicit_shift49_golden(orc, kats):
    # coefficient form with shift 49 instead of 7 (test_ntt_cpu.cpp:182-263):
    # INTT, scale coefficient i by 49^i, zero pad, NTT on 32 points.
    n = 16
    a = [1, 1]
    for i in range(2, n):
        a.append((a[-1] + a[-2]) % P)
    coeffs = orc.ntt(np.array(a, dtype=np.uint64).reshape(n, 1), inverse=True)[:, 0]
    ext = np.zeros((32, 1), dtype=np.uint64)
    g = 1
    for i in range(n):
        ext[i, 0] = _pmul(int(coeffs[i]), g)
        g = _pmul(g, 49)
    out = orc.ntt(ext)[:, 0]
    assert [int(v) for v in out] == kats["lde_shift49_fib_16_32"]


@pytest.mark.parametrize("case", [(16, 64, 1), (16, 32, 4), (64, 256, 8)])
def test_lde_horner(orc, case):
    # LDE(NTT(coeffs)) = coeffs evaluated on 7 * w_NExt^j (test_ntt_cpu.cpp:415-471)
    n, next_, ncols = case
    coeff = np.array([[((k * ncols + c + 1) * 1000003) % P for c in range(ncols)] for k in range(n)],
                     dtype=np.uint64)
    evals = orc.ntt(coeff)
    lde = orc.lde(evals, next_.bit_length() - 1)
    w = orc.root_of_unity(next_.bit_length() - 1)
    wj = 1
    for j in range(next_):
        x = _pmul(7, wj)
        for c in range(ncols):
            v = int(coeff[n - 1, c])
            for k in range(n - 2, -1, -1):
                v = (v * x + int(coeff[k, c])) % P
            assert int(lde[j, c]) == v
        wj = _pmul(wj, w)


def test_ntt_roundtrip(orc):
    x = oracle.random_field((1 << 9, 3), 99)
    assert (orc.ntt(orc.ntt(x), inverse=True) == x).all()


def _seeded(kats, max_nbits):
    return [c for c in kats["seeded_commits"] if c["nBits"] <= max_nbits]


def test_seeded_roots_oracle(orc, kats):
    for c in _seeded(kats, 16):
        trace = oracle.random_field((1 << c["nBits"], c["nCols"]), c["seed"])
        root, lde, tree = orc.commit(trace, c["nBitsExt"], c["arity"])
        assert [int(v) for v in root] == c["root"], c
        assert digest(lde) == c["lde_sha256"], c
        assert digest(tree) == c["tree_sha256"], c


def test_seeded_roots_reference_build(refcpu, kats):
    for c in _seeded(kats, 12):
        trace = oracle.random_field((1 << c["nBits"], c["nCols"]), c["seed"])
        root, lde, _ = refcpu.commit(trace, c["nBitsExt"], c["arity"])
        assert [int(v) for v in root] == c["root"], c


def test_oracle_matches_reference_build_random(orc, refcpu):
    for seed, (nb, nbe, nc, ar) in enumerate([(7, 8, 11, 4), (7, 9, 20, 3), (6, 7, 30, 2)]):
        trace = oracle.random_field((1 << nb, nc), 500 + seed)
        r1, l1, t1 = orc.commit(trace, nbe, ar)
        r2, l2, t2 = refcpu.commit(trace, nbe, ar)
        assert (l1 == l2).all() and (t1 == t2).all()


def test_tree_num_elements(orc):
    for n in [1, 2, 3, 4, 5, 16, 17, 1 << 10, (1 << 10) + 3]:
        for ar in (2, 3, 4):
            assert oracle.tree_num_elements(n, ar) == orc.lib.orc_tree_num_elements(n, ar)


# ---- Poseidon1 (hash family 1): the reference's test_poseidon_cpu.cpp goldens ----

def _fib(n):
    out = [0, 1]
    while len(out) < n:
        out.append((out[-1] + out[-2]) % oracle.P)
    return np.array(out[:n], dtype=np.uint64)


def _fib_rows(ncols, nrows):
    """buildMerkleInput (test_poseidon_cpu.cpp:175-186): rows 0 and 1 are 1..ncols, then
    row_j = row_{j-2} + row_{j-1}."""
    m = np.zeros((nrows, ncols), dtype=object)
    m[0] = m[1] = np.arange(1, ncols + 1)
    for j in range(2, nrows):
        m[j] = (m[j - 2] + m[j - 1]) % oracle.P
    return m.astype(np.uint64)


@pytest.fixture(scope="module")
def orc1():
    return oracle.Oracle(family=1)


def test_p1_permute_goldens(orc1, kats):
    g = kats["poseidon1"]
    assert [int(v) for v in orc1.permute(_fib(12))] == g["PERMUTE_FIB_W12_GOLDEN"]
    assert [int(v) for v in orc1.permute(np.zeros(12, dtype=np.uint64))] == g["PERMUTE_ZERO_W12_GOLDEN"]
    assert [int(v) for v in orc1.permute(np.arange(8, dtype=np.uint64))] == g["PERMUTE_W8_POSEIDON1_PLONKY3_GOLDEN"]
    assert [int(v) for v in orc1.permute(np.arange(16, dtype=np.uint64))] == g["PERMUTE_W16_POSEIDON1_GOLDEN"]


def test_p1_linear_hash_golden(orc1, kats):
    out = orc1.linear_hash(12, _fib(128))
    assert [int(v) for v in out] == kats["poseidon1"]["LINEAR_HASH_FIB128_W12_GOLDEN"]
    assert not orc1.linear_hash(12, np.zeros(0, dtype=np.uint64)).any()


def test_p1_merkletree_goldens(orc1, kats):
    g = kats["poseidon1"]
    tree = orc1.merkletree_w(12, _fib_rows(128, 64), 2)
    assert [int(v) for v in tree[-4:]] == g["MERKLE_BINARY_FIB128x64_ROOT"]
    tree = orc1.merkletree_w(12, np.zeros((64, 0), dtype=np.uint64), 2)
    assert [int(v) for v in tree[-4:]] == g["MERKLE_BINARY_EMPTY_64_ROOT"]
    tree = orc1.merkletree_w(12, np.zeros((1 << 17, 0), dtype=np.uint64), 2)
    assert [int(v) for v in tree[-4:]] == g["MERKLE_BINARY_EMPTY_POT17_ROOT"]


def test_p1_seeded_roots(orc1, kats):
    for case in kats["seeded_commits_poseidon1"]:
        trace = oracle.random_field((1 << case["nBits"], case["nCols"]), case["seed"])
        root, _, tree = orc1.commit(trace, case["nBitsExt"], case["arity"])
        assert [int(v) for v in root] == case["root"], case
        assert digest(tree) == case["tree_sha256"]


def test_p1_oracle_matches_reference_build(orc1):
    ref1 = oracle.RefCPU(family=1)
    for w in (8, 12, 16):
        st = oracle.random_field((w,), 100 + w)
        assert (orc1.permute(st) == ref1.permute(st)).all()
        data = oracle.random_field((3 * w + 1,), 200 + w)
        assert (orc1.linear_hash(w, data) == ref1.linear_hash(w, data)).all()
    m = oracle.random_field((100, 9), 7)
    for w, arity in ((8, 2), (12, 2), (12, 3), (16, 2), (16, 3), (16, 4)):
        assert (orc1.merkletree_w(w, m, arity) == ref1.merkletree_w(w, m, arity)).all(), (w, arity)


@pytest.mark.parametrize("family", [1, 2])
@pytest.mark.parametrize("arity", [2, 3, 4])
def test_group_proof_roundtrip(family, arity):
    """Oracle openings hash back to the root (both hash families); llv > 0 stops early."""
    o = oracle.Oracle(family=family)
    m = oracle.random_field((200, 9), 31 + arity)
    tree = o.merkletree(m, arity)
    for row in (0, 57, 199):
        proof = o.group_proof(m, tree, arity, row)
        assert (o.root_from_proof(proof, 9, 200, arity, row) == tree[-4:]).all()
        short = o.group_proof(m, tree, arity, row, llv=2)
        assert len(short) < len(proof) and (short == proof[:len(short)]).all()


def test_commit_q_coefficient_chunks(orc):
    """computeQ restated: chunk p of each limb's coefficients, times (7^-1)^(N*p), is column
    p*qDim + k of cmQ, which has degree < N."""
    nb, nbe, qdeg, qdim = 4, 6, 3, 3
    q = oracle.random_field((1 << nbe, qdim), 5)
    _, cmq, _ = orc.commit_q(q, nb, nbe, qdeg, qdim, 4)
    co = orc.ntt(cmq, inverse=True)
    assert not co[1 << nb:].any()
    qc = orc.ntt(q, inverse=True)
    P = oracle.P
    shift_in = pow(pow(7, P - 2, P), 1 << nb, P)
    for p in range(qdeg):
        S = pow(shift_in, p, P)
        for i in range(1 << nb):
            for k in range(qdim):
                assert int(co[i, p * qdim + k]) == int(qc[p * (1 << nb) + i, k]) * S % P


def test_commit_q_oracle_matches_reference_fixtures(orc, kats):
    """The oracle's computeQ restatement against the reference's own NTT/field code run on the
    same seeded q (ref_commit_q, written into the fixtures by make_golden.py)."""
    assert len(kats["seeded_q_commits"]) >= 5
    for c in kats["seeded_q_commits"]:
        q = oracle.random_field((1 << c["nBitsExt"], c["qDim"]), c["seed"])
        root, cmq, tree = orc.commit_q(q, c["nBits"], c["nBitsExt"], c["qDeg"], c["qDim"], c["arity"])
        assert [int(v) for v in root] == c["root"]
        assert digest(oracle.Oracle.canon(cmq)) == c["cmq_sha256"]
        assert digest(tree) == c["tree_sha256"]


def test_commit_q_reference_build_reproduces_fixture(refcpu, kats):
    c = kats["seeded_q_commits"][0]
    q = oracle.random_field((1 << c["nBitsExt"], c["qDim"]), c["seed"])
    root, cmq, _ = refcpu.commit_q(q, c["nBits"], c["nBitsExt"], c["qDeg"], c["qDim"], c["arity"])
    assert [int(v) for v in root] == c["root"] and [int(v) for v in cmq[1]] == c["cmq_row1"]


def test_seeded_generator_matches_product_host_generator(pkg, refcpu):
    """The full-size fixtures are built from ref_fill_random; the GPU tests and bench.py fill the same
    trace with the product's generator.  Both must give the same words (this call is host-only)."""
    for n, seed in ((1, 0), (1000, 1000), (1 << 16, 7), (4099, 2 ** 63 + 5)):
        assert (refcpu.fill_random(n, seed) == pkg.fill_random_host(n, seed)).all()


def test_full_size_fixture_file():
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "full_size.json")
    with open(path) as f:
        shapes = {s["name"]: s for s in json.load(f)["shapes"]}
    assert set(shapes) >= {"c2", "c4"}
    assert (shapes["c2"]["nBits"], shapes["c2"]["nBitsExt"], shapes["c2"]["nCols"]) == (22, 23, 256)
    assert (shapes["c4"]["nBits"], shapes["c4"]["nBitsExt"], shapes["c4"]["nCols"]) == (20, 22, 780)
    for s in shapes.values():
        assert len(s["root"]) == 4 and all(0 <= v < P for v in s["root"])
        assert s["tree_words"] == oracle.tree_num_elements(1 << s["nBitsExt"], s["arity"])
        assert len(s["sample_row0"]) == s["nCols"] and s["sample_rows"][0] == 0
