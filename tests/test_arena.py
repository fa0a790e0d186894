"""The commit server's budget allocator (csrc/arena.h, BlockMap), on the host.

A randomized sequence of takes and gives over a small range must never hand out overlapping or
out-of-range blocks, must keep free + live words equal to the range, must never keep two adjacent
free ranges apart, and must end as one free range when every block is back.  Best fit: a request
goes to the smallest free range that holds it.  Compiled with the host C++ compiler (no device).
"""
import os
import shutil
import subprocess
import tempfile

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "arena.h"

static int fail(const char *what, int step) { std::printf("FAIL %s at step %d\n", what, step); return 1; }

int main(int argc, char **argv)
{
    const uint64_t total = 32 * 4096;
    BlockMap m(total + 17);  // the range is rounded down to whole units
    if (m.total() != total) return fail("total", -1);
    std::mt19937_64 rng(std::strtoull(argv[1], nullptr, 10));
    struct Live { uint64_t off, w; };
    std::vector<Live> live;
    for (int step = 0; step < 200000; step++) {
        if (live.empty() || rng() % 2) {
            const uint64_t w = rng() % 4 == 0 ? 0 : 1 + rng() % (rng() % 2 ? 64 : 4000);
            // the best fit by brute force: the smallest free range that holds round(w)
            uint64_t want = BlockMap::NONE, best_len = ~0ull;
            for (auto &f : m.free_ranges())
                if (f.second >= BlockMap::round(w) && f.second < best_len) { best_len = f.second; want = f.first; }
            const uint64_t off = m.take(w);
            if (off != want) return fail("best fit", step);
            if (off == BlockMap::NONE) continue;
            if (off % BlockMap::UNIT || off + BlockMap::round(w) > total) return fail("range", step);
            for (auto &l : live)
                if (off < l.off + BlockMap::round(l.w) && l.off < off + BlockMap::round(w)) return fail("overlap", step);
            live.push_back({off, w});
        } else {
            const size_t i = rng() % live.size();
            m.give(live[i].off, live[i].w);
            live[i] = live.back();
            live.pop_back();
        }
        uint64_t used = 0, freew = 0, prev_end = ~0ull;
        for (auto &l : live) used += BlockMap::round(l.w);
        for (auto &f : m.free_ranges()) {
            if (f.first == prev_end) return fail("uncoalesced", step);
            prev_end = f.first + f.second;
            freew += f.second;
        }
        if (used + freew != total) return fail("accounting", step);
    }
    for (auto &l : live) m.give(l.off, l.w);
    if (m.free_ranges().size() != 1 || m.free_ranges().begin()->second != total) return fail("final", -1);
    std::printf("ok\n");
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    cxx = shutil.which("g++") or shutil.which("c++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    d = tempfile.mkdtemp()
    src = os.path.join(d, "arena_check.cpp")
    with open(src, "w") as f:
        f.write(DRIVER)
    exe = os.path.join(d, "arena_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(REPO, "pil2-proofman_b200", "csrc"), src, "-o", exe],
                   check=True, capture_output=True, timeout=120)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_block_map_randomized(driver, seed):
    r = subprocess.run([driver, str(seed)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
