// FRI query openings read from the resident LDE and Merkle tree.
//
// One opening is MerkleTreeGL::getGroupProof (merkleTreeGL.cpp:145-175): the queried row's
// nCols values, then for every tree level from the leaves up the (arity - 1) sibling digests
// of the path node in child order (4 words each), until the root — or, with
// last_level_verification = llv > 0, until a level holds at most arity^llv nodes (those are
// checked against the level itself, MerkleTreeGL::getLevel).  The GPU reference gathers the
// same words from its column-major buffers (getTreeTracePols / genMerkleProof,
// starks_gpu.cu:903-1042).
//
// Layout here: LDE column-major (col * NExt + row), tree in the reference buffer layout
// (levels padded to a multiple of the arity).  One CTA per query; its threads stride over the
// opening's words, so the column gather (one word per column, NExt apart) runs in parallel.
#pragma once
#include <stdint.h>

namespace query {

// sibling levels of an opening (genMerkleProof's recursion depth)
__host__ __device__ inline uint64_t proof_levels(uint64_t nrows, uint64_t arity, uint64_t llv)
{
    uint64_t stop = 1;
    for (uint64_t i = 0; i < llv; i++) stop *= arity;
    uint64_t levels = 0, n = nrows;
    while (llv ? (n > stop) : (n > 1)) {
        levels++;
        n = (n + arity - 1) / arity;
    }
    return levels;
}

inline uint64_t proof_words(uint64_t nrows, uint64_t ncols, uint64_t arity, uint64_t llv)
{
    return ncols + proof_levels(nrows, arity, llv) * (arity - 1) * 4;
}

__global__ void __launch_bounds__(256) openings_kernel(uint64_t *__restrict__ out, const uint64_t *__restrict__ lde,
                                                       uint64_t nrows, uint64_t ncols,
                                                       const uint64_t *__restrict__ tree, uint64_t arity,
                                                       uint64_t levels, const uint64_t *__restrict__ rows,
                                                       uint64_t words)
{
    const uint64_t q = blockIdx.x;
    const uint64_t row = rows[q];
    uint64_t *o = out + q * words;
    if (row >= nrows) {  // out-of-range query: an all-zero opening (the host checks rows first)
        for (uint64_t j = threadIdx.x; j < words; j += blockDim.x) o[j] = 0;
        return;
    }
    for (uint64_t c = threadIdx.x; c < ncols; c += blockDim.x) o[c] = lde[c * nrows + row];
    const uint64_t per_level = (arity - 1) * 4;
    for (uint64_t k = threadIdx.x; k < levels * per_level; k += blockDim.x) {
        const uint64_t level = k / per_level, within = k % per_level;
        // walk up to `level`: node index and buffer offset (in digests) of that level
        uint64_t idx = row, offset = 0, n = nrows;
        for (uint64_t l = 0; l < level; l++) {
            const uint64_t next = (n + arity - 1) / arity;
            offset += next * arity;
            idx /= arity;
            n = next;
        }
        const uint64_t cur = idx % arity, si = idx - cur;
        uint64_t s = within / 4;  // s-th sibling in child order, skipping the path node
        if (s >= cur) s++;
        o[ncols + k] = tree[(offset + si + s) * 4 + (within & 3)];
    }
}

}  // namespace query
