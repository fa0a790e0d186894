/*
 * pil2_b200 — B200-native (sm_100a) commit path for pil2-proofman:
 * low-degree extension of Goldilocks columns + Poseidon2 Merkle tree to one root.
 *
 * Two groups of entry points, all extern "C", plain pointers and sizes:
 *
 *  1. The reference's own C ABI for the commit path, same names and signatures as
 *     pil2-stark/src/api/starks_api.hpp, so the Rust crates (provers/starks-lib-c,
 *     ffi_starks.rs) can bind this library in place of libstarksgpu.a.  stark_info_new parses
 *     the setup's starkinfo JSON into this library's StarkInfo, and commit_witness takes
 *     proofman's SetupC {p_stark_info, p_expressions_bin} exactly as the reference does.
 *
 *  2. A native API on device or host buffers (prefix b200_), used by the tests and the
 *     benchmark, and by callers that manage device memory themselves.
 *
 * Conventions
 *  - Field elements are uint64_t; results are canonical (x mod p, p = 2^64 - 2^32 + 1);
 *    inputs may be any 64-bit value (taken mod p).
 *  - Device LDE buffers are column-major: element (row, col) at col*NExt + row
 *    (the reference GPU layout, goldilocks_trace_layout.cuh:14-46).  Traces given as
 *    row-major are element (row, col) at row*nCols + col (the reference CPU layout).
 *  - Tree buffers have b200_tree_num_elements(rows, arity) words in the reference layout
 *    (poseidon2_goldilocks.cpp:129-175); the root is the last 4 words.
 *  - Arity 2, 3, 4 uses Poseidon2 width 8, 12, 16 (merkleTreeGL.cpp:316-336).
 *  - int-returning functions return 0 on success and a negative B200_E* code on error;
 *    b200_last_error() describes the last error of the calling thread.  No entry point
 *    aborts the process.
 */
#ifndef PIL2_B200_H
#define PIL2_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B200_OK 0
#define B200_EINVAL -1    /* bad shape / argument */
#define B200_ECUDA -2     /* CUDA runtime error */
#define B200_ENOMEM -3    /* device or host allocation failed */
#define B200_EFAMILY -4   /* hash family not set, or not Poseidon2 */
#define B200_EBUSY -5     /* no admission (serving queue full / budget) */
#define B200_ETIMEOUT -6  /* bounded wait expired */

/* ------------------------------------------------------------------------------------
 * 1. Reference C ABI (pil2-stark/src/api/starks_api.hpp)
 * ------------------------------------------------------------------------------------ */

/* proofman's SetupC (common/src/setup.rs:45-57), which the reference reads as
 * SetupCtx {StarkInfo &, ExpressionsBin &} (starkpil/setup_ctx.hpp:200-207).  p_stark_info comes from
 * stark_info_new (or b200_stark_shape_new); p_expressions_bin is not read on the commit path. */
typedef struct B200SetupC {
    void *p_stark_info;
    void *p_expressions_bin;
} B200SetupC;

/* Layout of StepsParams (starkpil/steps.hpp:6-20 == common/src/air_instance.rs:20-33);
 * commit_witness reads `trace` (host, row-major N x nCols). */
typedef struct B200StepsParams {
    uint64_t *trace;
    uint64_t *aux_trace;
    uint64_t *publicInputs;
    uint64_t *proofValues;
    uint64_t *challenges;
    uint64_t *airgroupValues;
    uint64_t *airValues;
    uint64_t *evals;
    uint64_t *xDivXSub;
    uint64_t *pConstPolsAddress;
    uint64_t *pConstPolsExtendedTreeAddress;
    uint64_t *pCustomCommitsFixed;
} B200StepsParams;

/* starks_api.hpp:28 — 1 = Poseidon1 (PoseidonGoldilocks<W>), 2 = Poseidon2 (Poseidon2Goldilocks<W>);
 * the reference-ABI commit entries hash with the family set here.  Must be called before them,
 * once per process (a different second value is refused, as in the reference). */
void set_hash_family(uint8_t fam);

/* starks_api.hpp:37,48 — parse a starkinfo JSON file (StarkInfo::load, stark_info.cpp:24-263) for the
 * fields the commit path and the prover-buffer map need: starkStruct (nBits, nBitsExt, nQueries,
 * merkleTreeArity, lastLevelVerification, verificationHashType, steps), nConstants, nPublics, nStages,
 * qDeg, qDim, customCommits, the value/challenge/evaluation/opening maps' sizes and mapSectionsN; then
 * lay out the prover buffer as StarkInfo::setMapOffsets does for the given flags.  Returns NULL (and
 * b200_last_error) on a missing file or malformed JSON instead of exiting. */
void *stark_info_new(char *filename, bool recursive_final, bool recursive, bool verify_constraints, bool verify,
                     bool gpu, bool preallocate, bool single_use);
void stark_info_free(void *pStarkInfo);
/* starks_api.hpp:44-46: mapTotalN, mapTotalNCustomCommitsFixed, mapTotalNContributions of the map */
uint64_t get_map_total_n(void *pStarkInfo);
uint64_t get_map_total_n_custom_commits_fixed(void *pStarkInfo);
uint64_t get_map_total_n_contributions(void *pStarkInfo);
/* starks_api.hpp:59 — N * nConstants */
uint64_t get_const_size(void *pStarkInfo);

/* starks_api.hpp:52 — per-device set-up (twiddle/coset tables, kernel attributes) for the
 * current device.  The Poseidon2 constants are compiled in. */
void init_gpu_setup(uint64_t arity);

/* starks_api.hpp:190,193 — device commit buffers: a pool of streams, each owning device
 * buffers for one commit (grown on demand, kept resident until the slot is reused so the
 * LDE and tree can be read by later queries).  node_rank/node_size/numa_nodes are accepted
 * for signature compatibility; this library uses the current device. */
void *gen_device_buffers(uint32_t node_rank, uint32_t node_size, const int32_t *numa_nodes, uint32_t arity,
                         uint32_t max_n_bits_ext);
void free_device_buffers(void *d_buffers);

/* starks_api.hpp:198 — resize the stream pool to n_streams slots (other args accepted for
 * signature compatibility).  Returns the number of slots. */
uint64_t gen_device_streams(void *d_buffers, uint64_t n_streams, uint64_t n_recursive_streams,
                            const uint64_t *auxTraceSizes, uint64_t maxSizeProverBufferAggregation,
                            uint64_t maxProofSize, uint64_t merkleTreeArity);

/* starks_api.hpp:96 — synchronous: LDE + tree of a row-major host buffer N x nCols; writes the
 * 4-word root.  If bufferFile is a non-empty path, writes [root 32 B][source N*nCols words]
 * [LDE NExt*nCols words][tree nodes] with source and LDE column-major, as the reference's GPU
 * backend does (starks_api.cu:1867-1930). */
void write_custom_commit(void *root, uint64_t arity, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                         void *d_buffers, void *buffer, char *bufferFile);

/* starks_api.hpp:98 — asynchronous stage-1 commit of params->trace (host, row-major N x
 * mapSectionsN["cm1"]).  pSetupCtx points to a B200SetupC.  The commit lands in the stream's prover
 * buffer at the StarkInfo's mapOffsets, as commit_witness_gpu does (starks_api.cu:1599-1795): the
 * column-major trace at ("cm1", false), the LDE at ("cm1", true), the tree at ("mt1", true)
 * (b200_commit_buffers_aux).  Returns the stream slot id (or UINT64_MAX on error); the root is
 * written to `root` when get_stream_proofs / get_stream_proofs_non_blocking harvests the slot.  The
 * host trace may be reused after wait_trace_h2d_done(d_buffers, slot). */
uint64_t commit_witness(void *pSetupCtx, void *params, uint64_t instanceId, uint64_t airgroupId, uint64_t airId,
                        void *root, void *d_buffers, char *customCommitsFixedPath);

/* starks_api.hpp:127-128 — harvest finished commits (blocking: all in flight). */
void get_stream_proofs(void *d_buffers);
void get_stream_proofs_non_blocking(void *d_buffers);

/* starks_api.hpp:42 */
void wait_trace_h2d_done(void *d_buffers, uint64_t stream_id);

/* starks_api.hpp:40-41 (GPU backend: register_host_memory_gpu, starks_api.cu:86-104) — page-lock
 * a caller-owned host range (whole pages) for direct DMA, as proofman's memory handler does for
 * its trace buffers (common/src/memory_handler.rs); the trace copies of commit_witness then run at
 * full PCIe rate.  Returns 1 when pinned, 0 otherwise (null, empty, or the driver refused);
 * unregister ignores errors. */
uint32_t register_host_memory(void *ptr, uint64_t size);
void unregister_host_memory(void *ptr);

/* starks_api.hpp:61 — pStarkInfo from stark_info_new (or b200_stark_shape_new).  Host const pols
 * N x nConstants row-major in, host tree out: [LDE column-major NExt*nConstants][nodes]
 * (calculate_const_tree_gpu, starks_api.cu:1932-1980).  unified_buffer_gpu, if non-NULL, is a
 * device buffer of at least that many words used instead of a temporary allocation. */
void calculate_const_tree(void *pStarkInfo, void *pConstPolsAddress, void *pConstTree, void *unified_buffer_gpu);

/* starks_api.hpp:58 — words in the const tree buffer above */
uint64_t get_const_tree_size(void *pStarkInfo);

/* starks_api.hpp:230 — this library is GPU-only: returns true, ignores false */
bool set_gpu_mode(bool use_gpu);

/* ------------------------------------------------------------------------------------
 * 2. Native API
 * ------------------------------------------------------------------------------------ */

/* A StarkInfo built from the commit's four numbers instead of a starkinfo file (nCols is both
 * mapSectionsN["cm1"] and nConstants), with the stage-1 contribution buffer laid out as
 * [cm1 extended][tree][cm1].  Use it as p_stark_info or pStarkInfo; free with b200_stark_shape_free. */
void *b200_stark_shape_new(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity);
void b200_stark_shape_free(void *shape);
/* mapOffsets[(section, extended != 0)] of a StarkInfo, UINT64_MAX if absent */
uint64_t b200_stark_info_offset(void *pStarkInfo, const char *section, int extended);
/* a parsed field by name: nBits, nBitsExt, merkleTreeArity, lastLevelVerification, nConstants, nQueries,
 * qDeg, qDim, or mapSectionsN.<section>; UINT64_MAX if unknown */
uint64_t b200_stark_info_value(void *pStarkInfo, const char *name);
/* the prover buffer of stream slot stream_id (device pointer) and the words its last commit used */
int b200_commit_buffers_aux(void *d_buffers, uint64_t stream_id, uint64_t **d_aux, uint64_t *words);

const char *b200_last_error(void);
/* last error recorded on a d_buffers object by a void reference-ABI call (0 if none) */
int b200_buffers_error(void *d_buffers);

/* sets up the given device (tables, attributes); called implicitly by every entry point */
int b200_init(int device);
int b200_device_count(void);

uint64_t b200_tree_num_elements(uint64_t nrows, uint64_t arity);

/* Hash family of the native b200_* entry points: 1 = Poseidon1 (PoseidonGoldilocks<W>),
 * 2 = Poseidon2 (default), the values of set_hash_family (starks_api.hpp:28).  The reference
 * entry points follow set_hash_family, which may be set once per process; the native ones may
 * switch at any time (not while a call is running); a batched plan and a commit server keep
 * the family they were created under. */
int b200_set_native_hash_family(int family);
int b200_native_hash_family(void);
/* words of scratch the LDE needs (one column-major copy of the trace) */
uint64_t b200_lde_scratch_words(uint64_t nBits, uint64_t nCols);

/* Device-pointer API; stream is a cudaStream_t (NULL = legacy default stream).  All calls
 * are asynchronous on `stream` except where a host output is requested. */

/* LDE: d_lde column-major NExt x nCols; d_trace row-major (trace_rowmajor != 0) or column-major
 * with stride N; d_scratch holds b200_lde_scratch_words() words and overlaps neither. */
int b200_lde_device(uint64_t *d_lde, const uint64_t *d_trace, int trace_rowmajor, uint64_t nBits,
                    uint64_t nBitsExt, uint64_t nCols, uint64_t *d_scratch, void *stream);

/* The same LDE for callers that may not allocate device memory — a prover whose device
 * memory all comes from its own pool or budget (torch's caching allocator, a preallocated
 * arena), or a latency-critical loop that must not pay cudaMalloc's implicit device
 * synchronisation.  No counterpart in the reference (its LDE allocates or borrows a
 * buffer).  The scratch is a 64 MiB array inside this library's image, held by every GPU
 * that loads the library until exit: N * nCols must be <= 2^23 (larger shapes return
 * B200_EINVAL).  No cudaMalloc / cudaFree or other allocating call is made (with the
 * optional kernel timers off, the default).  The array is part of the library's device image:
 * the driver reserves its 64 MiB when it loads that image on a device, which with lazy module
 * loading (CUDA_MODULE_LOADING=LAZY) happens at the first call into the library there (this one,
 * b200_init or any other) — call b200_init(device) at set-up to pay it then.  The first call of
 * this entry point on a device resolves the array's device address and uploads the twiddle
 * tables; make that first call before any stream capture.  The address is kept per device for the
 * life of the process: cudaDeviceReset is not supported (nor is it for the library's other
 * per-device state).  All calls share the one array, which keeps the last call's contents
 * (nothing in it needs to start at zero): calls that overlap on the GPU — on different
 * streams or from different threads — race and must be serialised by the caller. */
int b200_lde_device_static_scratch(uint64_t *d_lde, const uint64_t *d_trace, int trace_rowmajor, uint64_t nBits,
                                   uint64_t nBitsExt, uint64_t nCols, void *stream);

/* Merkle tree (leaf sponge + levels) over element (row, col) = d_src[row*rs + col*cs]. */
int b200_merkletree_device(uint64_t *d_tree, const uint64_t *d_src, uint64_t rs, uint64_t cs, uint64_t nCols,
                           uint64_t nRows, uint64_t arity, void *stream);

/* LDE + tree.  If root_host is non-NULL, the root is copied there and the stream synchronised. */
int b200_commit_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree, const uint64_t *d_trace,
                       int trace_rowmajor, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t arity,
                       uint64_t *d_scratch, void *stream);

/* n independent Poseidon2 permutations of width 8/12/16 (d_in, d_out: n*width words). */
int b200_permute_device(uint64_t *d_out, const uint64_t *d_in, uint64_t n, uint64_t width, void *stream);

/* Host-buffer API (synchronous, allocates its own device memory): row-major trace in,
 * root out; lde_out (column-major NExt x nCols) and tree_out may be NULL. */
int b200_commit_host(uint64_t *root, uint64_t *lde_out, uint64_t *tree_out, const uint64_t *trace, uint64_t nBits,
                     uint64_t nBitsExt, uint64_t nCols, uint64_t arity);

/* Seeded synthetic field data: element i = the first splitmix64 output below p from the
 * stream keyed by (seed, i).  Host and device versions give identical values. */
int b200_fill_random_device(uint64_t *d_buf, uint64_t n, uint64_t seed, void *stream);
void b200_fill_random_host(uint64_t *buf, uint64_t n, uint64_t seed);

/* Rows of a resident LDE (query openings): out[i*nCols + c] = lde[c*NExt + rows[i]]. */
int b200_lde_rows_device(uint64_t *d_out, const uint64_t *d_lde, uint64_t NExt, uint64_t nCols,
                         const uint64_t *d_rows, uint64_t nrows_req, void *stream);

/* ---- Batched commit of many instances (device buffers) ---------------------------------
 * One plan covers a fixed set of instances (shapes and buffers).  A run performs, for all of
 * them together: one grouped transpose launch, one grouped launch per NTT window index, one
 * persistent leaf-sponge launch per arity (resident CTAs claim 128-row blocks of any instance
 * from a device counter), one grouped launch per tree level, one root gather.  With use_graph
 * the first run captures that sequence into a CUDA graph and later runs replay it (stream
 * must then be a created stream).  Results are bit-identical to b200_commit_device per
 * instance.  The batched counterpart of the reference's per-instance commit loop
 * (starks_api.cu:1599-1795 run once per instance on a stream from the pool). */
typedef struct B200BatchInstance {
    const uint64_t *d_trace; /* row-major N x nCols */
    uint64_t *d_scratch;     /* b200_lde_scratch_words(nBits, nCols) words */
    uint64_t *d_lde;         /* out: column-major NExt x nCols */
    uint64_t *d_tree;        /* out: b200_tree_num_elements(NExt, arity) words */
    uint64_t nBits, nBitsExt, nCols, arity;
} B200BatchInstance;

void *b200_batch_plan_new(const B200BatchInstance *inst, uint64_t n);
/* roots_host: n*4 words (may be NULL: then the call does not wait for the GPU) */
int b200_batch_plan_run(void *plan, uint64_t *roots_host, void *stream, int use_graph);
void b200_batch_plan_free(void *plan);
uint64_t b200_batch_plan_launches(void *plan);
int b200_commit_batch_device(const B200BatchInstance *inst, uint64_t n, uint64_t *roots_host, void *stream);

/* ---- Commit server (continuous batching) ------------------------------------------------
 * Requests (host row-major traces; pinned memory lets the copies overlap) are admitted as soon
 * as one of `slots` slots is free and the request's device buffers fit in `budget_bytes`, which
 * b200_server_new reserves on the device at once (one allocation, carved per request on the host;
 * NULL with B200_ENOMEM when it cannot be reserved); an admitted unit's host-to-device copy
 * overlaps the kernels of the units ahead of it (a large trace crosses in column blocks, each
 * extended as it lands), and the units' kernels run in admission order.  The small requests waiting
 * together (LDE of at most small_elems elements) are admitted as one batched unit (one
 * b200_batch_plan over all of them) and may pass waiting large requests, each of which is passed
 * at most four times.  The LDE and tree of a finished request stay on the device
 * (b200_server_buffers, for query reads) until b200_server_release; release them only after the
 * caller's own work on those buffers has completed, since the next admission may reuse them.
 * The reference's stream pool + selectStream + get_stream_proofs loop (starks_api.cu:1138-1170,
 * 2665-...) is the one-request-per-stream counterpart. */
void *b200_server_new(int device, uint64_t budget_bytes, uint32_t slots);
/* Before the first submit: batching 1 (default) as above, 0 = FIFO (every request a plain unit in
 * arrival order; the comparison point); small_elems (default 2^26) and max_batch (requests per
 * batched unit, default 64). */
int b200_server_configure(void *srv, int batching, uint64_t small_elems, uint32_t max_batch);
/* counters into out[0..n): plain units, batched units, requests in batched units, requests that
 * fit the budget but once found no contiguous block of it free (and waited), times a waiting
 * request was passed, microseconds the worker spent enqueueing units (allocations, copies,
 * launches), microseconds of that in allocations */
int b200_server_stats(void *srv, uint64_t *out, uint64_t n);
/* submission, admission and completion time of a request in ms since the server was created
 * (times3[1], times3[2] = -1 until reached) */
int b200_server_request_times(void *srv, int64_t id, double *times3);
/* device timeline of a completed request's unit in ms of device time since the server was created:
 * copies issued (the unit reached its stream), host-to-device copies done, kernels started (copies
 * done and the unit ahead finished), kernels done; -1 until the request completes */
int b200_server_request_gpu_times(void *srv, int64_t id, double *times4);
/* returns a request id > 0, or B200_EBUSY if the request can never fit the budget */
int64_t b200_server_submit(void *srv, const uint64_t *host_trace, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                           uint64_t arity, uint64_t *root_out);
/* 1 done (latency_ms = completion - submission), 0 queued or running, < 0 error */
int b200_server_status(void *srv, int64_t id, double *latency_ms);
int b200_server_wait_all(void *srv, uint64_t timeout_ms);
int b200_server_release(void *srv, int64_t id);
int b200_server_buffers(void *srv, int64_t id, uint64_t **d_lde, uint64_t **d_tree);
void b200_server_free(void *srv);

/* Names of the kernels this library launches (for test evidence), newline separated. */
const char *b200_kernel_names(void);

/* Kernel-category GPU timers (cudaEvent pairs on the launching stream; off by default).
 * Categories: 0 transpose, 1 ntt_inverse, 2 ntt_forward, 3 leaf_hash, 4 tree_levels.
 * b200_timing_get waits for the recorded events and returns the category's total ms and
 * the number of timed launch groups. */
void b200_timing_enable(int on);
void b200_timing_reset(void);
int b200_timing_get(int category, double *total_ms, uint64_t *count);
const char *b200_timing_name(int category);

/* Kernels launched by this library since the process started. */
uint64_t b200_launch_count(void);

/* Row-major -> column-major transposes: 1 (default) stages the tiles with the Tensor Memory
 * Accelerator where the source is 16-byte aligned with an even column count, 0 always uses the
 * thread-loaded shared-memory tiles.  Same values either way; returns the previous setting. */
int b200_set_transpose_tma(int on);
/* 1 if a TMA transpose tile copy did not land within the kernel's wait bound since the last call
 * (the flag is then reset), 0 otherwise, < 0 on a CUDA error. */
int b200_tma_wait_errors(void);

/* INT32 multiply-add throughput probe: `blocks` x 256 threads each run 8 independent
 * mad.lo/mad.hi chains of `iters` steps; returns the measured rate in G IMAD/s. */
int b200_probe_imad(uint64_t blocks, uint64_t iters, double *gimad_per_s);

/* ---- FRI query openings from the resident LDE and tree ----
 * One opening = MerkleTreeGL::getGroupProof (merkleTreeGL.cpp:145-175): the row's nCols values,
 * then per tree level the (arity-1) sibling digests of the path node in child order, up to the
 * root, or with last_level_verification = llv > 0 until a level holds <= arity^llv nodes.
 * Replaces the GPU reference's getTreeTracePols + genMerkleProof (starks_gpu.cu:903-1042).
 * d_lde column-major NExt x nCols, d_tree in the reference layout, d_rows nQueries row indices;
 * d_out receives nQueries x b200_query_proof_words() words. */
uint64_t b200_query_proof_words(uint64_t NExt, uint64_t nCols, uint64_t arity, uint64_t last_level_verification);
int b200_query_openings_device(uint64_t *d_out, const uint64_t *d_lde, uint64_t NExt, uint64_t nCols,
                               const uint64_t *d_tree, uint64_t arity, uint64_t last_level_verification,
                               const uint64_t *d_rows, uint64_t nQueries, void *stream);

/* ---- Q-stage commit (Starks::computeQ, starks.hpp:186-239; computeQColMajor,
 * ntt_goldilocks.cu:1515-1544) ----
 * d_q: qDim limb columns of NExt quotient evaluations (column-major, or row-major NExt x qDim);
 * d_cmq: column-major NExt x (qDeg*qDim), column p*qDim + k = chunk p of limb k extended;
 * d_tree: b200_tree_num_elements(NExt, arity) words; d_scratch: b200_q_scratch_words() words.
 * Requires qDeg <= NExt / N.  root_host (optional) receives the root after a stream sync. */
uint64_t b200_q_scratch_words(uint64_t nBitsExt, uint64_t qDim);
int b200_commit_q_device(uint64_t *root_host, uint64_t *d_cmq, uint64_t *d_tree, const uint64_t *d_q,
                         int q_rowmajor, uint64_t nBits, uint64_t nBitsExt, uint64_t qDeg, uint64_t qDim,
                         uint64_t arity, uint64_t *d_scratch, void *stream);

/* ---- LDE plan autotuner (no reference counterpart: the reference's NTT has a fixed plan) ----
 * b200_autotune_lde times the LDE of (nBits, nBitsExt) under each window plan on a probe of
 * min(nCols, 64) columns and records the fastest for nCols' bucket; plain, batched and served
 * commits then use it.  Plans change speed only, never results.  The table can be read, set,
 * saved to and loaded from a text file. */
int b200_autotune_lde(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, double *best_ms, uint32_t *kfirst,
                      uint32_t *krest);
void b200_autotune_get(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint32_t *kfirst, uint32_t *krest);
void b200_autotune_set(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint32_t kfirst, uint32_t krest);
int b200_autotune_save(const char *path);
int b200_autotune_load(const char *path);

/* ---- packed-witness commit (PackedInfo + unpack, starks_gpu.cu:49-103; the packed branch of
 * commit_witness_gpu, starks_api.cu:1660-1676) ----
 * d_packed: N rows of words_per_row u64 words; column c takes the next col_bits[c] (1..64) bits
 * of its row, least significant first, straddling words.  col_bits is a host array.  Same
 * outputs as b200_commit_device on the unpacked trace. */
uint64_t b200_packed_words_per_row(const uint32_t *col_bits, uint64_t nCols);
int b200_commit_packed_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree, const uint64_t *d_packed,
                              uint64_t words_per_row, const uint32_t *col_bits, uint64_t nBits, uint64_t nBitsExt,
                              uint64_t nCols, uint64_t arity, uint64_t *d_scratch, void *stream);

/* ---- streaming slot commit of a bit-packed witness (commit_witness_streaming & co.,
 * starks_api.hpp:212-217; streamCommitPacked, goldilocks/src/stream_commit.cuh) ----
 * Columns are extended and absorbed RATE = 12 at a time into the row sponge (W16, arity 4), so
 * the NExt x nCols LDE is never materialised; the root equals the ordinary commit's.  nCols must
 * be 1..64 and nBitsExt > nBits (stream_commit_slot_bytes returns 0 otherwise).  The reference
 * entry points hash with Poseidon1 only (set_hash_family(1), else -15), own their slots
 * (configure_stream_commit_slots) and are synchronous.  Return codes: 0, -10 invalid shape or
 * widths, -11 no slots, -12 slot index, -13 slot too small, -14 paused.  colWidths: host array
 * of nCols u64 widths (1..64); packed: host rows of wordsPerRow u64 words. */
uint64_t stream_commit_slot_bytes(uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow);
void configure_stream_commit_slots(void *d_buffers, uint64_t nSlots, uint64_t slotBytes);
uint64_t get_stream_commit_slots(void *d_buffers);
uint64_t get_stream_commit_floor(void *d_buffers);
int64_t commit_witness_streaming(void *d_buffers, uint64_t slotIdx, uint64_t airgroupId, uint64_t airId, void *packed,
                                 uint64_t nBits, uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow,
                                 void *colWidths, void *root);
void stream_commit_pause(void);
/* Native form: caller-owned device slot of slot_words words (>= stream_commit_slot_bytes / 8),
 * the native hash family (b200_set_native_hash_family); synchronous on `stream`. */
int b200_stream_commit_packed(uint64_t *d_slot, uint64_t slot_words, const uint64_t *h_packed, uint64_t nBits,
                              uint64_t nBitsExt, uint64_t nCols, uint64_t wordsPerRow, const uint64_t *colWidths,
                              uint64_t *root, void *stream);

/* ---- indexed witness (instruction table; unpack_indexed, starks_gpu.cu:125-185) ----
 * A row is a leading instruction index (index_bits) followed by the runtime columns; columns with
 * col_source[c] = 1 are read from entry `index` of the instruction table (words_per_entry words
 * per entry; an index past the table selects entry 0).  register_instruction_table
 * (starks_api.hpp:192) hands the table to the buffers object; b200_register_indexed_air stands in
 * for the setup's PackedInfo (which columns come from the table, the index width).  With both
 * registered for (airgroupId, airId), commit_witness_streaming commits that AIR's indexed rows
 * (-16 when the table is missing). */
void register_instruction_table(void *d_buffers, uint64_t airgroupId, uint64_t airId, uint64_t *table,
                                uint64_t num_entries, uint64_t words_per_entry);
int b200_register_indexed_air(void *d_buffers, uint64_t airgroupId, uint64_t airId, uint64_t nCols,
                              const uint8_t *col_source, uint64_t index_bits);
int b200_commit_indexed_device(uint64_t *root_host, uint64_t *d_lde, uint64_t *d_tree, const uint64_t *d_rows,
                               uint64_t words_per_row, const uint64_t *d_table, uint64_t num_entries,
                               uint64_t words_per_entry, uint64_t index_bits, const uint64_t *col_bits,
                               const uint8_t *col_source, uint64_t nBits, uint64_t nBitsExt, uint64_t nCols,
                               uint64_t arity, uint64_t *d_scratch, void *stream);
int b200_stream_commit_indexed(uint64_t *d_slot, uint64_t slot_words, const uint64_t *h_rows, uint64_t nBits,
                               uint64_t nBitsExt, uint64_t nCols, uint64_t words_per_row, const uint64_t *col_bits,
                               const uint8_t *col_source, uint64_t index_bits, const uint64_t *d_table,
                               uint64_t num_entries, uint64_t words_per_entry, uint64_t *root, void *stream);

/* MerkleTreeGL::getLevel (merkleTreeGL.cpp:84-101): the first level of <= arity^llv nodes, zero-filled
 * to arity^llv nodes (b200_tree_last_level_words words) — what llv-deep openings are checked against. */
uint64_t b200_tree_last_level_words(uint64_t arity, uint64_t last_level_verification);
int b200_tree_last_level_device(uint64_t *d_out, const uint64_t *d_tree, uint64_t NExt, uint64_t arity,
                                uint64_t last_level_verification, void *stream);
/* merkletreeReduce (Poseidon2Goldilocks<W>::merkletreeReduce, W = 4 * arity; native hash family):
 * the tree above n digests (4 words each) in d_tree (b200_tree_num_elements(n, arity) words). */
int b200_merkletree_reduce_device(uint64_t *root_host, const uint64_t *d_digests, uint64_t n, uint64_t arity,
                                  uint64_t *d_tree, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PIL2_B200_H */
