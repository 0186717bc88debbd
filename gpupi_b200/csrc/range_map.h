// Best-fit allocation of byte ranges inside one block, with freed neighbours
// coalesced: the host-side bookkeeping of the scratch arena (scratch.cu).
// Plain C++, no CUDA, so it is tested on its own.
#pragma once

#include <stddef.h>

#include <iterator>
#include <map>

namespace gpupi {

class RangeMap {
public:
    // The whole block [0, size) becomes one free range.
    void reset(size_t size) {
        free_at_.clear();
        free_by_size_.clear();
        if (size) insert(0, size);
    }
    // Offset of a free range of `size` bytes (the smallest that fits), or
    // false when none does.
    bool take(size_t size, size_t *offset) {
        auto it = free_by_size_.lower_bound(size);
        if (it == free_by_size_.end()) return false;
        const size_t have = it->first, off = it->second;
        erase(off, have);
        if (have > size) insert(off + size, have - size);
        *offset = off;
        return true;
    }
    // Returns [offset, offset + size) to the free ranges, merged with free
    // neighbours.
    void give(size_t offset, size_t size) { insert(offset, size); }
    size_t free_ranges() const { return free_at_.size(); }
    const std::map<size_t, size_t> &ranges() const { return free_at_; }

private:
    void erase(size_t off, size_t size) {
        free_at_.erase(off);
        auto r = free_by_size_.equal_range(size);
        for (auto it = r.first; it != r.second; ++it)
            if (it->second == off) {
                free_by_size_.erase(it);
                return;
            }
    }
    void insert(size_t off, size_t size) {
        auto next = free_at_.lower_bound(off);
        if (next != free_at_.end() && off + size == next->first) {
            const size_t noff = next->first, nsize = next->second;
            erase(noff, nsize);
            size += nsize;
        }
        auto it = free_at_.lower_bound(off);
        if (it != free_at_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == off) {
                const size_t poff = prev->first, psize = prev->second;
                erase(poff, psize);
                off = poff;
                size += psize;
            }
        }
        free_at_[off] = size;
        free_by_size_.emplace(size, off);
    }

    std::map<size_t, size_t> free_at_;            // offset -> size
    std::multimap<size_t, size_t> free_by_size_;  // size -> offset
};

}  // namespace gpupi
