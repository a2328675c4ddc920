// serve_arena.h - first-fit allocator over one reserved HBM range.
//
// The served form reserves its whole device budget once and carves every
// launch group's buffers out of it, so admission is a host-side decision
// ("does this group fit in what is free") and no cudaMalloc runs while
// requests are in flight.  Offsets only: the caller adds the range's base.
#pragma once

#include <cstdint>
#include <iterator>
#include <map>

namespace ma {

class OffsetArena {
  public:
    static constexpr uint64_t kAlign = 256;
    static constexpr uint64_t kFail = ~0ull;

    explicit OffsetArena(uint64_t capacity = 0) { reset(capacity); }

    void reset(uint64_t capacity) {
        free_.clear();
        used_ = 0;
        peak_ = 0;
        capacity_ = capacity & ~(kAlign - 1);
        if (capacity_) free_[0] = capacity_;
    }

    static uint64_t round_up(uint64_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

    // Offset of a block of at least n bytes (256-aligned), or kFail.
    uint64_t alloc(uint64_t n) {
        n = round_up(n ? n : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const uint64_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            used_ += n;
            if (used_ > peak_) peak_ = used_;
            return off;
        }
        return kFail;
    }

    // Returns a block; neighbours merge so that the range never fragments
    // into more pieces than there are live blocks.
    void release(uint64_t off, uint64_t n) {
        n = round_up(n ? n : 1);
        used_ -= n;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && off + n == next->first) {
            n += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += n;
                return;
            }
        }
        free_[off] = n;
    }

    uint64_t largest_free() const {
        uint64_t m = 0;
        for (const auto& kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }
    uint64_t used() const { return used_; }
    uint64_t peak() const { return peak_; }
    uint64_t capacity() const { return capacity_; }
    size_t pieces() const { return free_.size(); }

  private:
    std::map<uint64_t, uint64_t> free_;  // offset -> length
    uint64_t capacity_ = 0, used_ = 0, peak_ = 0;
};

}  // namespace ma
