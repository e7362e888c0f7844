// The sketch server's host-side rules (shgemm_b200/csrc/server_host.hpp), run without a GPU.
//  - The offset allocator behind the server's arena against a map of 256-byte units:
//    every allocation lands where first fit over the free units says, never overlaps a live
//    block, the free byte count and the number of free runs match the map after every step,
//    and releasing everything leaves one run of the whole size.
//  - A table of the row chunks and tile counts of a set of requests, one line per chunk,
//    for tests/test_server_host.py to compare with its own statement of the rules.
// Prints "allocator ok" and the table; exits non-zero on the first disagreement.
#include "server_host.hpp"

#include <cstdio>
#include <random>
#include <vector>

using namespace shgemm_b200_server_host;

namespace {

struct Block {
    size_t off, bytes;
};

size_t units_of(size_t bytes) { return round_up(std::max<size_t>(bytes, 1)) / kAlign; }

int check_allocator(unsigned seed, size_t units, int steps) {
    OffsetAllocator a;
    a.reset(units * kAlign - 100);  // rounded up to whole units
    if (a.size() != units * kAlign || a.free_bytes() != a.size() || a.free_runs() != 1) {
        std::printf("reset: size %zu free %zu runs %zu\n", a.size(), a.free_bytes(), a.free_runs());
        return 1;
    }
    std::vector<char> used(units, 0);
    std::vector<Block> live;
    std::mt19937_64 rng(seed);
    for (int step = 0; step < steps; ++step) {
        const bool grow = live.empty() || rng() % 100 < 55;
        if (grow) {
            size_t bytes = 1 + rng() % (64 * kAlign);
            if (rng() % 50 == 0) bytes = 0;  // a zero-byte request still takes one unit
            const size_t need = units_of(bytes);
            size_t want = OffsetAllocator::kNone;
            for (size_t i = 0, run = 0; i < units; ++i) {
                run = used[i] ? 0 : run + 1;
                if (run == need) {
                    want = (i + 1 - need) * kAlign;
                    break;
                }
            }
            const size_t got = a.alloc(bytes);
            if (got != want) {
                std::printf("step %d: alloc(%zu) = %zu, first fit says %zu\n", step, bytes, got, want);
                return 2;
            }
            if (got == OffsetAllocator::kNone) continue;
            for (size_t u = got / kAlign; u < got / kAlign + need; ++u) used[u] = 1;
            live.push_back({got, bytes});
        } else {
            const size_t i = rng() % live.size();
            const Block b = live[i];
            a.release(b.off, b.bytes);
            for (size_t u = b.off / kAlign; u < b.off / kAlign + units_of(b.bytes); ++u) used[u] = 0;
            live[i] = live.back();
            live.pop_back();
        }
        size_t free_units = 0, runs = 0;
        for (size_t i = 0; i < units; ++i) {
            free_units += used[i] ? 0 : 1;
            runs += (!used[i] && (i == 0 || used[i - 1])) ? 1 : 0;
        }
        if (a.free_bytes() != free_units * kAlign || a.free_runs() != runs) {
            std::printf("step %d: free %zu bytes in %zu runs, the map has %zu in %zu\n", step, a.free_bytes(),
                        a.free_runs(), free_units * kAlign, runs);
            return 3;
        }
    }
    for (const Block& b : live) a.release(b.off, b.bytes);
    if (a.free_bytes() != a.size() || a.free_runs() != 1) {
        std::printf("after releasing all: free %zu of %zu in %zu runs\n", a.free_bytes(), a.size(), a.free_runs());
        return 4;
    }
    return 0;
}

}  // namespace

int main() {
    for (unsigned seed = 1; seed <= 4; ++seed) {
        const int rc = check_allocator(seed, seed == 1 ? 64 : 4096, 20000);
        if (rc) return rc;
    }
    std::printf("allocator ok\n");
    // m, n, draws, k: the served stream's extremes and values in between
    const size_t shapes[][4] = {{1024, 64, 4, 1024},    {65536, 256, 4, 16384}, {65536, 64, 4, 1024},
                                {40000, 128, 4, 9000},  {1000, 256, 1, 16384},  {300, 7, 3, 5},
                                {128, 256, 4, 16384},   {129, 256, 4, 16384},   {65535, 200, 2, 12345},
                                {50000, 256, 8, 16384}, {4096, 33, 4, 2048},    {70000, 1, 1, 1}};
    for (const auto& s : shapes) {
        const size_t m = s[0], n = s[1], k = s[3];
        const int draws = static_cast<int>(s[2]);
        for (size_t row = 0; row < m;) {
            const size_t rows = chunk_rows(m, row, n, draws, k);
            if (rows == 0) return 5;
            std::printf("chunk %zu %zu %d %zu %zu %zu %d\n", m, n, draws, k, row, rows,
                        piece_units(rows, n * static_cast<size_t>(draws)));
            row += rows;
        }
    }
    return 0;
}
