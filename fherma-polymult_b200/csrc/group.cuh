// Grouped launches: one launch of a stage kernel covers the blocks of many
// products (points of different N, q and K), the way a grouped GEMM covers many
// problems.  The table travels in kernel-parameter space (__grid_constant__),
// so a block finds its product with a few constant-bank loads and reads that
// product's DevPoint from there as a plain launch reads its own.
//
// Block b of a launch belongs to item i with first[i] <= b < first[i + 1]; its
// local index b - first[i] is split by the stage (prime, tile) or (operand,
// tile).  Items are ordered by the host (largest first), which also decides
// the order in which a persistent grid meets them.
#pragma once

#include "device.cuh"

#include <cstdint>

namespace fpm {

constexpr int kGroupMax = 64;   // items per grouped launch (table about 16 KB)

struct GroupItem {
    DevPoint d;
    const uint32_t* a;   // N x L limbs (decompose input)
    const uint32_t* b;
    uint32_t* A;         // K x N residues
    uint32_t* B;
    uint32_t* c;         // N x L limbs (CRT output)
    uint32_t j0;         // transform passes: the item covers primes j0 .. j0 + blocks / per - 1
};

struct GroupTable {
    uint32_t count;                   // items
    uint32_t total;                   // blocks over all items
    uint32_t first[kGroupMax + 1];    // first block of each item; first[count] = total
    GroupItem item[kGroupMax];
};

static_assert(sizeof(GroupTable) < 32000, "grouped launch table must fit kernel-parameter space");

// Item owning block b (binary search over the prefix table).
__device__ __forceinline__ uint32_t group_locate(const GroupTable& t, uint32_t b) {
    uint32_t lo = 0, hi = t.count;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (t.first[mid] <= b) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

}  // namespace fpm
