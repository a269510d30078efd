// Randomised check of ldp::Region (the serving loop's placement of job
// arenas in one device region) against a unit-by-unit model of the region.
// Prints "ok" or the first violation and exits non-zero.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "ldp_region.h"

namespace {

constexpr size_t kUnit = 256;

struct Block {
    size_t off, bytes;
};

int fail(const char* what, int seed, int step) {
    std::printf("seed %d step %d: %s\n", seed, step, what);
    return 1;
}

}  // namespace

int main() {
    for (int seed = 0; seed < 200; ++seed) {
        std::mt19937_64 rng((uint64_t)seed);
        const size_t units = 64 + rng() % 4000;
        ldp::Region r;
        r.reset(units * kUnit);
        std::vector<char> used(units, 0);   // the model: one flag per unit
        std::vector<Block> live;
        for (int step = 0; step < 2000; ++step) {
            const bool take = live.empty() || (rng() % 100) < 55;
            if (take) {
                // sizes from one unit to a third of the region, not always
                // whole units (the allocator rounds up to 256 bytes)
                const size_t bytes = 1 + rng() % (units * kUnit / 3);
                const size_t need = (bytes + kUnit - 1) / kUnit;
                // first fit in the model
                size_t want = ldp::Region::kNone;
                for (size_t u = 0, run = 0; u < units; ++u) {
                    run = used[u] ? 0 : run + 1;
                    if (run == need) {
                        want = (u + 1 - need) * kUnit;
                        break;
                    }
                }
                const size_t got = r.take(bytes);
                if (got != want) return fail("offset differs from first fit", seed, step);
                if (got == ldp::Region::kNone) continue;
                if (got % kUnit) return fail("unaligned offset", seed, step);
                for (size_t u = got / kUnit; u < got / kUnit + need; ++u) used[u] = 1;
                live.push_back({got, bytes});
            } else {
                const size_t i = rng() % live.size();
                const Block b = live[i];
                live[i] = live.back();
                live.pop_back();
                r.give(b.off, b.bytes);
                const size_t need = (b.bytes + kUnit - 1) / kUnit;
                for (size_t u = b.off / kUnit; u < b.off / kUnit + need; ++u) used[u] = 0;
            }
            size_t free_units = 0, runs = 0;
            for (size_t u = 0; u < units; ++u) {
                free_units += !used[u];
                runs += !used[u] && (u == 0 || used[u - 1]);
            }
            if (r.free_bytes() != free_units * kUnit) return fail("free bytes differ", seed, step);
            // neighbours merge: one free block per run of free units
            if (r.free_blocks() != runs) return fail("free blocks not coalesced", seed, step);
        }
        for (const Block& b : live) r.give(b.off, b.bytes);
        if (r.free_blocks() != 1 || r.free_bytes() != units * kUnit) return fail("region not whole at the end", seed, -1);
    }
    std::printf("ok\n");
    return 0;
}
