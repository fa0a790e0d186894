"""Batched commit (grouped kernels, persistent leaf scheduler, CUDA graph) and the commit server.

Both must give, for every instance, exactly the plain path's LDE, tree and root (bit-exact;
integer field arithmetic), whether an instance runs alone or among others.
"""
import ctypes
import time

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


SHAPES = [  # (nBits, nBitsExt, nCols, arity): uneven rows, columns, blowups and arities
    (10, 11, 37, 4), (13, 15, 5, 4), (8, 9, 200, 4), (12, 13, 16, 3), (14, 15, 24, 4), (6, 8, 3, 2),
    (11, 11, 9, 4), (3, 4, 1, 4), (16, 17, 12, 4), (9, 12, 2, 4),
]


def _alloc(torch, pkg, shapes):
    bufs = []
    descs = (pkg.BatchInstance * len(shapes))()
    for j, (nb, nbe, nc, ar) in enumerate(shapes):
        N, NExt = 1 << nb, 1 << nbe
        t = {
            "trace": torch.empty(max(1, N * nc), dtype=torch.int64, device="cuda"),
            "scratch": torch.empty(max(1, N * nc), dtype=torch.int64, device="cuda"),
            "lde": torch.full((max(1, NExt * nc),), -1, dtype=torch.int64, device="cuda"),
            "tree": torch.full((pkg.tree_num_elements(NExt, ar),), -1, dtype=torch.int64, device="cuda"),
        }
        pkg.fill_random_device(t["trace"], N * nc, 700 + j)
        d = descs[j]
        d.d_trace, d.d_scratch, d.d_lde, d.d_tree = (t[k].data_ptr() for k in ("trace", "scratch", "lde", "tree"))
        d.nBits, d.nBitsExt, d.nCols, d.arity = nb, nbe, nc, ar
        bufs.append(t)
    torch.cuda.synchronize()
    return bufs, descs


def test_batch_matches_plain_and_oracle(pkg, torch_cuda, orc):
    torch = torch_cuda
    pkg.init(0)
    lib = pkg.load()
    bufs, descs = _alloc(torch, pkg, SHAPES)
    # plain results, instance by instance
    plain = []
    for j, (nb, nbe, nc, ar) in enumerate(SHAPES):
        t = bufs[j]
        lde = torch.empty_like(t["lde"])
        tree = torch.empty_like(t["tree"])
        scr = torch.empty_like(t["scratch"])
        root = pkg.commit_device(lde, tree, t["trace"], nb, nbe, nc, ar, scr)
        plain.append((root, lde.clone(), tree.clone()))
    stream = torch.cuda.Stream()
    plan = lib.b200_batch_plan_new(descs, len(SHAPES))
    assert plan, lib.b200_last_error()
    try:
        for use_graph in (0, 1, 1):  # direct, graph capture, graph replay
            roots = np.zeros((len(SHAPES), 4), dtype=np.uint64)
            for t in bufs:
                t["lde"].fill_(-1)
                t["tree"].fill_(-1)
            torch.cuda.synchronize()
            assert lib.b200_batch_plan_run(plan, roots.ctypes.data, stream.cuda_stream, use_graph) == 0
            for j in range(len(SHAPES)):
                assert (roots[j] == plain[j][0]).all(), (j, use_graph)
                assert torch.equal(bufs[j]["lde"], plain[j][1]), (j, use_graph)
                assert torch.equal(bufs[j]["tree"], plain[j][2]), (j, use_graph)
    finally:
        lib.b200_batch_plan_free(plan)
    # and the oracle agrees on a few of them
    for j in (0, 3, 5):
        nb, nbe, nc, ar = SHAPES[j]
        trace = bufs[j]["trace"].cpu().numpy().view(np.uint64)[: (1 << nb) * nc].reshape(1 << nb, nc)
        assert (orc.commit(trace, nbe, ar)[0] == plain[j][0]).all()


def test_batch_with_large_instances_matches_plain(pkg, torch_cuda):
    """Instances whose windows or transpose cover >= 2^27 elements run as the plain path's own
    launches inside the batch (the rest stay grouped); every LDE word, tree node and root must
    still equal the plain path's, in direct runs and in graph capture and replay."""
    torch = torch_cuda
    pkg.init(0)
    lib = pkg.load()
    shapes = [(20, 21, 128, 4), (12, 13, 16, 3), (19, 21, 300, 4), (17, 18, 40, 4)]
    bufs, descs = _alloc(torch, pkg, shapes)
    plain = []
    for j, (nb, nbe, nc, ar) in enumerate(shapes):
        t = bufs[j]
        lde, tree, scr = torch.empty_like(t["lde"]), torch.empty_like(t["tree"]), torch.empty_like(t["scratch"])
        root = pkg.commit_device(lde, tree, t["trace"], nb, nbe, nc, ar, scr)
        plain.append((root, lde, tree))
        del scr
    stream = torch.cuda.Stream()
    plan = lib.b200_batch_plan_new(descs, len(shapes))
    assert plan, lib.b200_last_error()
    try:
        for use_graph in (0, 1, 1):
            roots = np.zeros((len(shapes), 4), dtype=np.uint64)
            for t in bufs:
                t["lde"].fill_(-1)
                t["tree"].fill_(-1)
            torch.cuda.synchronize()
            assert lib.b200_batch_plan_run(plan, roots.ctypes.data, stream.cuda_stream, use_graph) == 0
            for j in range(len(shapes)):
                assert (roots[j] == plain[j][0]).all(), (j, use_graph)
                assert torch.equal(bufs[j]["lde"], plain[j][1]), (j, use_graph)
                assert torch.equal(bufs[j]["tree"], plain[j][2]), (j, use_graph)
    finally:
        lib.b200_batch_plan_free(plan)


def test_one_shot_batch_entry(pkg, torch_cuda):
    torch = torch_cuda
    lib = pkg.load()
    shapes = SHAPES[:4]
    bufs, descs = _alloc(torch, pkg, shapes)
    roots = np.zeros((len(shapes), 4), dtype=np.uint64)
    assert lib.b200_commit_batch_device(descs, len(shapes), roots.ctypes.data, None) == 0
    for j, (nb, nbe, nc, ar) in enumerate(shapes):
        t = bufs[j]
        r = pkg.commit_device(torch.empty_like(t["lde"]), torch.empty_like(t["tree"]), t["trace"], nb, nbe, nc, ar,
                              torch.empty_like(t["scratch"]))
        assert (roots[j] == r).all()


@pytest.mark.parametrize("mode,small", [(1, 1 << 26), (1, 1 << 17), (0, 1 << 26)])
def test_server_alone_equals_in_the_mix(pkg, torch_cuda, mode, small):
    """Each request's root is the same served alone and served among overlapping requests: with
    continuous batching (small requests admitted together share one batched unit; with the lower
    threshold the larger ones run as plain units beside them) and in FIFO mode.  Plain units of
    2^16 rows and >= 128 columns cross in column blocks extended as they land, the first request
    (on an idle device) with its rows hashed in chunks meanwhile."""
    lib = pkg.load()
    # the last two cross in column blocks when they run as plain units (2^16 rows, >= 128 columns)
    shapes = [(12, 13, 40, 4), (14, 15, 9, 4), (10, 12, 100, 3), (15, 16, 30, 4), (9, 10, 5, 2), (13, 14, 64, 4),
              (16, 17, 24, 4), (16, 17, 200, 4), (16, 18, 130, 3)]
    traces = [oracle.random_field((1 << nb, nc), 42 + i) for i, (nb, nbe, nc, ar) in enumerate(shapes)]
    alone = [pkg.commit_host(tr, nbe, ar)[0] for tr, (nb, nbe, nc, ar) in zip(traces, shapes)]
    srv = lib.b200_server_new(0, 8 << 30, 4)
    assert srv, lib.b200_last_error()
    try:
        assert lib.b200_server_configure(srv, mode, small, 64) == 0, lib.b200_last_error()
        ids, outs = [], []
        for rep in range(3):  # all requests in flight together, three times over
            for i, (nb, nbe, nc, ar) in enumerate(shapes):
                out = np.zeros(4, dtype=np.uint64)
                rid = lib.b200_server_submit(srv, traces[i].ctypes.data, nb, nbe, nc, ar, out.ctypes.data)
                assert rid > 0, lib.b200_last_error()
                ids.append((i, rid))
                outs.append(out)
        assert lib.b200_server_wait_all(srv, 60000) == 0, lib.b200_last_error()
        lat = ctypes.c_double()
        g = (ctypes.c_double * 4)()
        spans = set()
        for (i, rid), out in zip(ids, outs):
            assert lib.b200_server_status(srv, rid, ctypes.byref(lat)) == 1
            assert lat.value > 0
            assert (out == alone[i]).all(), i
            # device timeline: issued <= kernels started <= kernels done, and the copies done after
            # issue and before the kernels end (a plain unit's kernels start on its first column
            # block, so they may start before the last block has landed)
            assert lib.b200_server_request_gpu_times(srv, rid, g) == 0
            eps = 1e-3
            assert 0 <= g[0] <= g[2] + eps and g[2] <= g[3] + eps, list(g)
            assert g[0] <= g[1] + eps and g[1] <= g[3] + eps, list(g)
            spans.add((g[2], g[3]))
            # the LDE stays resident until release
            d_lde = ctypes.c_void_p()
            d_tree = ctypes.c_void_p()
            assert lib.b200_server_buffers(srv, rid, ctypes.byref(d_lde), ctypes.byref(d_tree)) == 0
            assert d_lde.value and d_tree.value
            assert lib.b200_server_release(srv, rid) == 0
        # the units' kernels run one after another, in admission order
        spans = sorted(spans)
        assert all(nxt[0] >= prev[1] - 1e-3 for prev, nxt in zip(spans, spans[1:])), spans
        # an oversized request is refused, not queued forever
        assert lib.b200_server_submit(srv, traces[0].ctypes.data, 24, 26, 64, 4, None) == pkg.B200_EBUSY
        st = (ctypes.c_uint64 * 5)()
        assert lib.b200_server_stats(srv, st, 5) == 0
        plain, batched, in_batches = st[0], st[1], st[2]
        assert plain + in_batches == 3 * len(shapes)
        if mode == 0:
            assert batched == 0
        # configuring after the first submit is refused
        assert lib.b200_server_configure(srv, 1, 1 << 20, 8) == pkg.B200_EBUSY
    finally:
        lib.b200_server_free(srv)


def test_server_batches_small_requests(pkg, torch_cuda):
    """Requests queued together while the server is busy are admitted as one batched unit."""
    lib = pkg.load()
    nb, nbe, nc = 11, 12, 20
    traces = [oracle.random_field((1 << nb, nc), 70 + i) for i in range(12)]
    want = [oracle.Oracle().commit(t, nbe, 4)[0] for t in traces]
    srv = lib.b200_server_new(0, 4 << 30, 1)  # one slot: the first request runs, the rest queue
    assert srv
    try:
        outs, ids = [], []
        for t in traces:
            out = np.zeros(4, dtype=np.uint64)
            ids.append(lib.b200_server_submit(srv, t.ctypes.data, nb, nbe, nc, 4, out.ctypes.data))
            outs.append(out)
        assert lib.b200_server_wait_all(srv, 60000) == 0, lib.b200_last_error()
        for out, w in zip(outs, want):
            assert (out == w).all()
        st = (ctypes.c_uint64 * 5)()
        lib.b200_server_stats(srv, st, 5)
        assert st[1] >= 1 and st[2] >= 2, list(st)
    finally:
        lib.b200_server_free(srv)


def test_server_admission_respects_budget(pkg, torch_cuda):
    """With a budget that fits one request at a time, requests still all complete, in order."""
    lib = pkg.load()
    nb, nbe, nc = 12, 13, 32
    per = 8 * (2 * (1 << nb) * nc + (1 << nbe) * nc + pkg.tree_num_elements(1 << nbe, 4))
    srv = lib.b200_server_new(0, int(per * 1.5), 4)
    assert srv
    try:
        trace = oracle.random_field((1 << nb, nc), 5)
        want = pkg.commit_host(trace, nbe, 4)[0]
        outs, ids = [], []
        for _ in range(5):
            out = np.zeros(4, dtype=np.uint64)
            ids.append(lib.b200_server_submit(srv, trace.ctypes.data, nb, nbe, nc, 4, out.ctypes.data))
            outs.append(out)
        t0 = time.time()
        while time.time() - t0 < 60:
            done = [lib.b200_server_status(srv, i, None) for i in ids]
            for i, d in zip(ids, done):
                if d == 1:
                    lib.b200_server_release(srv, i)  # frees the resident LDE so the next one is admitted
            if all(d == 1 for d in done):
                break
            time.sleep(0.005)
        assert all(lib.b200_server_status(srv, i, None) == 1 for i in ids)
        for out in outs:
            assert (out == want).all()
    finally:
        lib.b200_server_free(srv)
