#!/usr/bin/env python3
"""Write tests/golden/reference_kats.json: the known-answer vectors that pin the oracle.

Two sources, both from the reference (run here, where it is mounted):

1. The reference's own golden constants, read as text from its test sources:
   * pil2-stark/src/goldilocks/tests/test_helpers.hpp:17-66
     (Poseidon2 permute / permuteTrunc W4..W16 on input 0..W-1, linearHash W8/12/16
     on input 1..20, merkletreeReduce W12 arity 3 on digests 1..12)
   * pil2-stark/src/goldilocks/tests/test_ntt_cpu.cpp:182-263 (LDE with an explicit
     coset shift 49 of a Fibonacci column, N=16 -> 32) and :264-350 / :351-412
     (LDE_block / extendePol: 8 Fibonacci-like columns, N=16 -> 32, column 0 values).
   * pil2-stark/src/goldilocks/tests/test_poseidon_cpu.cpp:56-90,361-395 (Poseidon1: W12
     permute of a Fibonacci / zero state, W12 linearHash of 128 Fibonacci words, W12 arity-2
     merkletree roots of a 128 x 64 Fibonacci matrix and of 0-column matrices with 64 and 2^17
     rows, W8 permute of 0..7 (plonky3 cross-check), W16 permute of 0..15).
2. Outputs of the reference CPU implementation itself (NTT_Goldilocks::LDE and
   Poseidon2Goldilocks<W>::merkletree, compiled unmodified by oracle/Makefile) on
   seeded inputs: Merkle roots and an LDE digest per shape; and the Q-stage commit
   (Starks::computeQ, starks.hpp:186-239: NTT_Goldilocks::INTT over NExt, the chunk scaling by
   (shift^-1)^(N*p), NTT_Goldilocks::NTT, Poseidon2 tree) as ref_commit_q in
   oracle/ref_wrapper.cpp runs it on the reference's NTT and field code.

Usage (needs the reference checkout, found as oracle.reference_root() finds it, and
`make -C oracle ref`):  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
import oracle  # noqa: E402

REF = os.path.join(oracle.reference_root() or "reference", "pil2-stark", "src", "goldilocks", "tests")

# seeded shapes pinned by the reference CPU path: (nBits, nBitsExt, ncols, arity, seed).
# NExt = 4 is left out: there NTT_Goldilocks::NTT_iters clamps nphase to 2 (ntt_goldilocks.cpp:67-72),
# which sends reversePermutation into its in-place branch (:325-362); with extension > 1 that
# branch swaps some row pairs twice and reads rows past N, so its output is schedule-dependent.
# N = 1 (nBits = 0) is left out too: the reference CPU build corrupts its heap on it.
SEEDED = [
    (4, 5, 8, 4, 1),
    (6, 7, 1, 4, 2),
    (6, 8, 5, 4, 3),
    (8, 9, 12, 4, 4),
    (8, 9, 13, 4, 5),
    (8, 10, 24, 3, 6),
    (8, 9, 7, 2, 7),
    (10, 11, 32, 4, 8),
    (10, 11, 32, 3, 9),
    (12, 13, 3, 4, 10),
    (3, 4, 1, 4, 11),
    (2, 3, 2, 4, 12),
    (1, 3, 3, 4, 13),
    (1, 4, 5, 3, 14),
    (5, 5, 9, 4, 15),
    (16, 17, 32, 4, 1601),   # the CPU-runnable single-AIR case: 2^16 x 32, blowup 2
    (16, 17, 32, 3, 1602),
]


# seeded Poseidon1 (hash family 1) commits, W = 4 * arity as MerkleTreeGL picks it
SEEDED_P1 = [
    (4, 5, 8, 4, 21),
    (6, 7, 13, 3, 22),
    (8, 9, 7, 2, 23),
    (10, 11, 32, 4, 24),
    (12, 14, 12, 4, 25),
]


# seeded Q-stage commits: (nBits, nBitsExt, qDeg, qDim, arity, seed); qDim 3 is the cubic extension
# the reference's computeQ assumes (FIELD_EXTENSION), qDeg up to NExt / N
SEEDED_Q = [
    (4, 6, 3, 3, 4, 41),
    (6, 7, 2, 3, 4, 42),
    (8, 10, 4, 3, 3, 43),
    (10, 11, 1, 3, 2, 44),
    (5, 9, 16, 3, 4, 45),
    (12, 14, 3, 3, 4, 46),
    (14, 15, 2, 3, 4, 47),
]


def parse_helpers(text):
    out = {}
    for m in re.finditer(r"constexpr uint64_t (\w+)\[\d+\]\s*=\s*\{(.*?)\};", text, re.S):
        out[m.group(1)] = [int(v, 16) for v in re.findall(r"0x[0-9a-fA-F]+", m.group(2))]
    return out


def parse_lde_test(text, name):
    body = text.split("TEST(GOLDILOCKS_TEST, %s)" % name, 1)[1].split("TEST(", 1)[0]
    vals = re.findall(r"ASSERT_EQ\(Goldilocks::toU64\(a\[(\d+)(?: \* NUM_COLUMNS)?\]\), 0X([0-9A-Fa-f]+)\)", body)
    return [int(v, 16) for _, v in sorted(vals, key=lambda t: int(t[0]))]


def parse_poseidon1(text):
    out = {}
    for m in re.finditer(r"constexpr uint64_t (\w+)\[\w+\]\s*=\s*\{(.*?)\};", text, re.S):
        out[m.group(1)] = [int(v, 0) for v in re.findall(r"0[xX][0-9a-fA-F]+|\d+", m.group(2))]
    return out


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def main():
    with open(os.path.join(REF, "test_helpers.hpp")) as f:
        helpers = parse_helpers(f.read())
    with open(os.path.join(REF, "test_ntt_cpu.cpp")) as f:
        ntt_text = f.read()
    with open(os.path.join(REF, "test_poseidon_cpu.cpp")) as f:
        p1 = parse_poseidon1(f.read())
    for name, n in (("PERMUTE_FIB_W12_GOLDEN", 12), ("PERMUTE_ZERO_W12_GOLDEN", 12),
                    ("LINEAR_HASH_FIB128_W12_GOLDEN", 4), ("MERKLE_BINARY_FIB128x64_ROOT", 4),
                    ("MERKLE_BINARY_EMPTY_64_ROOT", 4), ("MERKLE_BINARY_EMPTY_POT17_ROOT", 4),
                    ("PERMUTE_W8_POSEIDON1_PLONKY3_GOLDEN", 8), ("PERMUTE_W16_POSEIDON1_GOLDEN", 16)):
        assert len(p1[name]) == n, name
    kats = {
        "source": "reference test sources (test_helpers.hpp, test_ntt_cpu.cpp) and the reference CPU build",
        "poseidon2": helpers,
        "poseidon1": p1,
        "lde_shift49_fib_16_32": parse_lde_test(ntt_text, "LDE"),
        "lde_block_16_32_col0": parse_lde_test(ntt_text, "LDE_block"),
        "extendePol_16_32_col0": parse_lde_test(ntt_text, "extendePol"),
    }
    assert len(kats["lde_shift49_fib_16_32"]) == 32
    assert kats["lde_block_16_32_col0"] == kats["extendePol_16_32_col0"]

    ref = oracle.RefCPU()
    seeded = []
    for nbits, nbits_ext, ncols, arity, seed in SEEDED:
        trace = oracle.random_field((1 << nbits, ncols), seed)
        root, lde, tree = ref.commit(trace, nbits_ext, arity)
        seeded.append({
            "nBits": nbits, "nBitsExt": nbits_ext, "nCols": ncols, "arity": arity, "seed": seed,
            "root": [int(v) for v in root],
            "lde_sha256": digest(lde),
            "tree_sha256": digest(tree),
            "lde_row0": [int(v) for v in lde[0]],
        })
        print("seeded", nbits, nbits_ext, ncols, arity, [hex(int(v)) for v in root])
    kats["seeded_commits"] = seeded
    ref1 = oracle.RefCPU(family=1)
    seeded1 = []
    for nbits, nbits_ext, ncols, arity, seed in SEEDED_P1:
        trace = oracle.random_field((1 << nbits, ncols), seed)
        root, lde, tree = ref1.commit(trace, nbits_ext, arity)
        seeded1.append({"nBits": nbits, "nBitsExt": nbits_ext, "nCols": ncols, "arity": arity, "seed": seed,
                        "root": [int(v) for v in root], "tree_sha256": digest(tree)})
        print("seeded poseidon1", nbits, nbits_ext, ncols, arity, [hex(int(v)) for v in root])
    kats["seeded_commits_poseidon1"] = seeded1
    seeded_q = []
    for nbits, nbits_ext, qdeg, qdim, arity, seed in SEEDED_Q:
        q = oracle.random_field((1 << nbits_ext, qdim), seed)
        root, cmq, tree = ref.commit_q(q, nbits, nbits_ext, qdeg, qdim, arity)
        seeded_q.append({"nBits": nbits, "nBitsExt": nbits_ext, "qDeg": qdeg, "qDim": qdim, "arity": arity,
                         "seed": seed, "root": [int(v) for v in root], "cmq_sha256": digest(cmq),
                         "tree_sha256": digest(tree), "cmq_row1": [int(v) for v in cmq[1]]})
        print("seeded Q", nbits, nbits_ext, qdeg, qdim, arity, [hex(int(v)) for v in root])
    kats["seeded_q_commits"] = seeded_q
    kats["seeded_generator"] = "oracle.random_field: numpy PCG64(seed), uniform u64 rejected unless < p, row-major"
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote reference_kats.json")


if __name__ == "__main__":
    main()
