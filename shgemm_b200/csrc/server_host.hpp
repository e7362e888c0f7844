// Host-side bookkeeping of the sketch server (shgemm_server.cpp), kept free of CUDA calls so
// that it builds and is tested with a plain C++ compiler: the first-fit offset allocator
// behind the server's device arena, and the rules that cut a large request into row chunks
// and count the tiles a launch makes of one.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <map>

namespace shgemm_b200_server_host {

constexpr size_t kAlign = 256;
inline size_t round_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator of offsets in [0, size()), in multiples of kAlign; a released block
// merges with free neighbours, so the free list is always the maximal free runs.
class OffsetAllocator {
   public:
    static constexpr size_t kNone = SIZE_MAX;

    void reset(size_t bytes) {
        size_ = round_up(bytes);
        free_.clear();
        if (size_) free_[0] = size_;
    }
    size_t size() const { return size_; }

    // Offset of `bytes` (rounded up, at least one unit) at the lowest free run that holds
    // them, or kNone.
    size_t alloc(size_t bytes) {
        bytes = round_up(std::max<size_t>(bytes, 1));
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, rest = it->second - bytes;
            free_.erase(it);
            if (rest) free_[off + bytes] = rest;
            return off;
        }
        return kNone;
    }

    // Returns a block from alloc() with the same size argument.
    void release(size_t off, size_t bytes) {
        bytes = round_up(std::max<size_t>(bytes, 1));
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

    size_t free_bytes() const {
        size_t s = 0;
        for (const auto& kv : free_) s += kv.second;
        return s;
    }
    size_t free_runs() const { return free_.size(); }

   private:
    size_t size_ = 0;
    std::map<size_t, size_t> free_;  // offset -> bytes
};

// A launch holds at most this many tiles.
constexpr int kMaxUnitsPerLaunch = 1 << 16;
// Work of one chunk of a large request, 2 m n k: ~1.6 ms on a B200 in TF32.
constexpr double kChunkFlops = 4e11;

// Rows of the next chunk of a request of m rows (n columns per draw, `draws` draws, depth k)
// whose first `row_next` rows are handed out: all that is left, or a multiple of 128 near
// kChunkFlops (at least 128).
inline size_t chunk_rows(size_t m, size_t row_next, size_t n, int draws, size_t k) {
    const size_t left = m - row_next;
    const double per_row = 2.0 * static_cast<double>(n) * draws * static_cast<double>(k);
    size_t rows = static_cast<size_t>(kChunkFlops / per_row) / 128 * 128;
    rows = std::max<size_t>(rows, 128);
    return rows >= left ? left : rows;
}

// Tiles a launch makes of `rows` rows and `cols` columns: 128-row tiles, tile N the smallest
// power of two in [32, 256] that covers cols (capped at 2^30).
inline int piece_units(size_t rows, size_t cols) {
    size_t bn = 32;
    while (bn < 256 && bn < cols) bn *= 2;
    return static_cast<int>(std::min<size_t>(((rows + 127) / 128) * ((cols + bn - 1) / bn), size_t(1) << 30));
}

}  // namespace shgemm_b200_server_host
