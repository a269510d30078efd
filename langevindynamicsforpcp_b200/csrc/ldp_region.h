// ldp_region.h -- first-fit placement of blocks in one region (host side).
//
// The serving loop allocates its memory budget once, as one device region,
// and places each admitted job's arena in it with this allocator: no device
// allocation per job.  Plain C++ (no CUDA), so the CPU tests exercise it.
#pragma once
#include <cstddef>
#include <iterator>
#include <map>

namespace ldp {

// First-fit placement of job arenas in one device region, with coalescing
// of free neighbours.  Offsets and sizes are multiples of 256 bytes.
class Region {
   public:
    void reset(size_t cap) {
        free_.clear();
        if (cap) free_[0] = cap;
    }
    // Offset of a free block of `bytes`, or kNone.
    size_t take(size_t bytes) {
        bytes = (bytes + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, left = it->second - bytes;
            free_.erase(it);
            if (left) free_[off + bytes] = left;
            return off;
        }
        return kNone;
    }
    void give(size_t off, size_t bytes) {
        bytes = (bytes + 255) & ~(size_t)255;
        auto nx = free_.lower_bound(off);
        if (nx != free_.end() && off + bytes == nx->first) {
            bytes += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                pv->second += bytes;
                return;
            }
        }
        free_[off] = bytes;
    }
    size_t free_bytes() const {
        size_t n = 0;
        for (const auto& kv : free_) n += kv.second;
        return n;
    }
    size_t free_blocks() const { return free_.size(); }
    static constexpr size_t kNone = ~(size_t)0;

   private:
    std::map<size_t, size_t> free_;   // offset -> size
};

}  // namespace ldp
