// kp_range_alloc.h -- first-fit allocator of integer ranges [0, capacity),
// host side.  The serving loop places each admitted job's ray records and
// outputs with it (ray ids index the record pool; output units are 256-byte
// blocks of the device output arena).  Freed ranges coalesce with their
// neighbours.
#pragma once

#include <iterator>
#include <map>

namespace kp {

class RangeAllocator {
public:
    explicit RangeAllocator(long long capacity = 0) { reset(capacity); }

    void reset(long long capacity) {
        free_.clear();
        capacity_ = capacity;
        used_ = 0;
        if (capacity > 0) free_[0] = capacity;
    }

    // Start of a free range of n units, or -1.
    long long alloc(long long n) {
        if (n <= 0) return -1;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const long long start = it->first;
            const long long left = it->second - n;
            free_.erase(it);
            if (left > 0) free_[start + n] = left;
            used_ += n;
            return start;
        }
        return -1;
    }

    void release(long long start, long long n) {
        if (n <= 0) return;
        used_ -= n;
        auto next = free_.lower_bound(start);
        long long s = start, len = n;
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == s) {
                s = prev->first;
                len += prev->second;
                free_.erase(prev);
            }
        }
        if (next != free_.end() && s + len == next->first) {
            len += next->second;
            free_.erase(next);
        }
        free_[s] = len;
    }

    long long capacity() const { return capacity_; }
    long long used() const { return used_; }
    long long largest_free() const {
        long long best = 0;
        for (const auto& kv : free_) best = kv.second > best ? kv.second : best;
        return best;
    }
    size_t fragments() const { return free_.size(); }

private:
    std::map<long long, long long> free_;  // start -> length
    long long capacity_ = 0;
    long long used_ = 0;
};

}  // namespace kp
