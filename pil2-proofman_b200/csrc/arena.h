// Best-fit block map over a range of 64-bit words (host bookkeeping only; no device calls), the
// allocator behind the commit server's device-memory budget.  Blocks are whole 256-byte units
// (32 words); free ranges are kept coalesced, so after every block is given back the map is one
// free range again.
#pragma once
#include <cstdint>
#include <iterator>
#include <map>

class BlockMap {
  public:
    static constexpr uint64_t NONE = ~0ull;
    static constexpr uint64_t UNIT = 32;  // words per 256 bytes

    explicit BlockMap(uint64_t words = 0) { reset(words); }
    void reset(uint64_t words)
    {
        free_.clear();
        total_ = words / UNIT * UNIT;
        if (total_) free_[0] = total_;
    }
    static uint64_t round(uint64_t w) { return (w ? w + UNIT - 1 : UNIT) / UNIT * UNIT; }
    uint64_t total() const { return total_; }

    // offset of a block of at least w words (the smallest free range that holds it), or NONE
    uint64_t take(uint64_t w)
    {
        w = round(w);
        auto best = free_.end();
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= w && (best == free_.end() || it->second < best->second)) best = it;
        if (best == free_.end()) return NONE;
        const uint64_t off = best->first, len = best->second;
        free_.erase(best);
        if (len > w) free_[off + w] = len - w;
        return off;
    }

    // the block taken at `off` for w words back to the free ranges, merged with its neighbours
    void give(uint64_t off, uint64_t w)
    {
        w = round(w);
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + w == next->first) {
            w += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += w;
                return;
            }
        }
        free_[off] = w;
    }

    const std::map<uint64_t, uint64_t> &free_ranges() const { return free_; }

  private:
    std::map<uint64_t, uint64_t> free_;  // offset -> length (words)
    uint64_t total_ = 0;
};
