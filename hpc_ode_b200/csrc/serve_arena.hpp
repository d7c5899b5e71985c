// First-fit range allocator over one pre-allocated device region.
//
// The request loop (serve.cu) reserves its whole device budget once and hands
// each admitted request one contiguous range of it, so admission is a host-side
// bookkeeping decision ("does the request's footprint fit in what is free?")
// and no cudaMalloc/cudaFree happens while kernels run.  Offsets only: the
// allocator never touches device memory, so it is plain C++ and testable on a
// CPU.
#pragma once

#include <cstddef>
#include <iterator>
#include <map>

namespace b200 {

class RangeArena {
public:
    static constexpr size_t kAlign = 256;

    explicit RangeArena(size_t capacity = 0) { reset(capacity); }

    void reset(size_t capacity) {
        cap_ = capacity / kAlign * kAlign;
        free_.clear();
        if (cap_) free_[0] = cap_;
        used_ = 0;
        peak_ = 0;
    }

    static size_t round_up(size_t bytes) { return (bytes + kAlign - 1) / kAlign * kAlign; }

    // First free range that holds `bytes` (rounded up to kAlign); returns false
    // when none does.
    bool alloc(size_t bytes, size_t* offset) {
        const size_t need = round_up(bytes ? bytes : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < need) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > need) free_[off + need] = len - need;
            used_ += need;
            if (used_ > peak_) peak_ = used_;
            *offset = off;
            return true;
        }
        return false;
    }

    // Returns [offset, offset + round_up(bytes)) and merges it with free neighbours.
    void release(size_t offset, size_t bytes) {
        size_t len = round_up(bytes ? bytes : 1);
        used_ -= len;
        auto next = free_.lower_bound(offset);
        if (next != free_.end() && offset + len == next->first) {
            len += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == offset) {
                prev->second += len;
                return;
            }
        }
        free_[offset] = len;
    }

    size_t capacity() const { return cap_; }
    size_t used() const { return used_; }
    size_t peak() const { return peak_; }
    size_t free_ranges() const { return free_.size(); }
    size_t largest_free() const {
        size_t m = 0;
        for (const auto& kv : free_)
            if (kv.second > m) m = kv.second;
        return m;
    }

private:
    size_t cap_ = 0, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;   // offset -> length
};

}  // namespace b200
