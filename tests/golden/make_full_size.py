#!/usr/bin/env python3
"""Write tests/golden/full_size.json: reference-CPU commits at the benchmarked full sizes.

The reference's own CPU implementation (NTT_Goldilocks::LDE + Poseidon2Goldilocks<16>::merkletree, or
PoseidonGoldilocks<16>::merkletree for hash family 1, compiled unmodified into oracle/_ref by
oracle/Makefile) commits the seeded traces of the two large single-instance workloads:

  c2            2^22 rows x 256 columns, blowup 2 (LDE 2^23 rows), arity 4
  c4            2^20 rows x 780 columns (600 base + 60 cubic-extension limbs), blowup 4 (LDE 2^22 rows), arity 4
  c2_poseidon1  the c2 trace hashed with Poseidon1 (hash family 1, the Rust side's default family)

Trace element i (row-major index) of seed s is the seeded rule shared by the oracle
(ref_fill_random) and the product (b200_fill_random_device / _host), so the GPU tests and
bench.py fill the same trace on the device without reading this script's inputs.  The LDE runs
column-blocked (nblock > 1 with a caller work buffer, ntt_goldilocks.cpp:217-255,369-397) so that
both shapes fit in ~40 GB of host memory; blocking changes the schedule, not the values.

Recorded per shape: the root, the SHA-256 of the whole canonical tree buffer (every leaf digest
and node), and sampled LDE rows (indices, the first sampled row in full, and the SHA-256 of all
sampled rows).  Usage (needs the reference checkout and `make -C oracle ref`; ~3 minutes and ~40 GB
of host memory on 8 cores):  python tests/golden/make_full_size.py [shape names to recompute]
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
import oracle  # noqa: E402

SHAPES = [
    # name, nBits, nBitsExt, nCols, arity, seed, nblock, hash family (2 Poseidon2, 1 Poseidon1)
    ("c2", 22, 23, 256, 4, 1000, 4, 2),
    ("c4", 20, 22, 780, 4, 1000, 4, 2),
    ("c2_poseidon1", 22, 23, 256, 4, 1000, 4, 1),
]
N_SAMPLE_ROWS = 32


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def sample_rows(nbits_ext, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    rows = np.unique(rng.integers(0, 1 << nbits_ext, size=N_SAMPLE_ROWS - 2))
    return sorted({0, (1 << nbits_ext) - 1, *[int(r) for r in rows]})


def main():
    refs = {f: oracle.RefCPU(threads=os.cpu_count(), family=f) for f in (1, 2)}
    out = {"source": "reference CPU build (oracle/_ref): NTT_Goldilocks::LDE + Poseidon2Goldilocks<16>::merkletree "
                     "(family 2) or PoseidonGoldilocks<16>::merkletree (family 1)",
           "generator": "ref_fill_random == b200_fill_random: splitmix64 keyed by (seed, row-major index), "
                        "rejection below p",
           "shapes": []}
    only = set(sys.argv[1:])  # optional: names of the shapes to (re)compute; the others are kept
    old = {}
    path = os.path.join(HERE, "full_size.json")
    if only and os.path.exists(path):
        with open(path) as f:
            old = {s["name"]: s for s in json.load(f)["shapes"]}
    for name, nb, nbe, nc, arity, seed, nblock, family in SHAPES:
        if only and name not in only and name in old:
            old[name].setdefault("family", family)
            out["shapes"].append(old[name])
            continue
        ref = refs[family]
        t0 = time.time()
        trace = ref.fill_random((1 << nb) * nc, seed).reshape(1 << nb, nc)
        lde = np.empty((1 << nbe, nc), dtype=np.uint64)
        buf = np.empty((1 << nbe) * -(-nc // nblock), dtype=np.uint64)
        ref.lde_raw(trace, nbe, out=lde, buffer=buf, nblock=nblock)
        del buf, trace
        tree = np.empty(oracle.tree_num_elements(1 << nbe, arity), dtype=np.uint64)
        ref.merkletree_raw(lde, arity, tree=tree)
        tree = oracle.RefCPU.canon(tree)
        rows = sample_rows(nbe, seed + 1)
        block = oracle.RefCPU.canon(lde[rows])
        del lde
        rec = {"name": name, "nBits": nb, "nBitsExt": nbe, "nCols": nc, "arity": arity, "seed": seed,
               "family": family,
               "root": [int(v) for v in tree[-4:]], "tree_sha256": digest(tree), "tree_words": int(tree.size),
               "sample_rows": rows, "sample_rows_sha256": digest(block), "sample_row0": [int(v) for v in block[0]],
               "seconds": round(time.time() - t0, 1)}
        del tree
        print(name, [hex(v) for v in rec["root"]], rec["seconds"], "s", flush=True)
        out["shapes"].append(rec)
    with open(os.path.join(HERE, "full_size.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote full_size.json")


if __name__ == "__main__":
    main()
