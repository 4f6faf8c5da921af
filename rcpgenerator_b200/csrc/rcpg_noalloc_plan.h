// Layout of the fixed scratch array of rcpg_pairs_full_noalloc: which byte
// ranges of the array hold which build array for a given N, ndim and row
// capacity, and how many cells the grid may use. Host-only arithmetic, shared
// by the entry point (rcpg_noalloc.cu) and the CPU test of the sizing.
#pragma once

#include <cstddef>
#include <cstdint>

namespace rcpg {

constexpr std::size_t kNoAllocScratchBytes = std::size_t{8} << 20;

// Offsets (bytes from the start of the array, each 256-byte aligned) of the
// arrays carved out of the scratch; ok = false when they do not fit.
struct NoAllocPlan {
    bool ok = false;
    std::size_t ctl, pos, spos, x_last, caps, cell_of, cell_rank, cell_list, work, nbr_cnt, nbr, scan_tmp;
    std::size_t cell_count, cell_start;
    std::uint32_t cell_capacity = 0;  // C_alloc: cells of the grid (the build coarsens to fit)
    std::size_t used = 0;             // bytes in use after the last array
};

// sizeof(DevCtl) is passed in so that this header needs no CUDA types.
inline NoAllocPlan plan_noalloc(std::uint64_t N, int ndim, std::uint32_t row_capacity, std::size_t ctl_bytes,
                                std::size_t cap = kNoAllocScratchBytes) {
    NoAllocPlan p;
    // N above the array size in bytes can never fit; refusing it first keeps
    // every product below within 64 bits
    if (N == 0 || N > cap || ndim < 2 || row_capacity == 0) return p;
    const std::uint64_t P = static_cast<std::uint64_t>((ndim + 2) & ~1);
    std::size_t used = 0;
    bool ok = true;
    auto take = [&](std::uint64_t count, std::size_t elem) -> std::size_t {
        const std::size_t off = (used + 255) & ~std::size_t{255};
        if (!ok || off > cap || count > (cap - off) / elem) {
            ok = false;
            return 0;
        }
        used = off + static_cast<std::size_t>(count) * elem;
        return off;
    };
    p.ctl = take(1, ctl_bytes);
    p.pos = take(N * P, 8);
    p.spos = take(N * P, 8);
    p.x_last = take(N * static_cast<std::uint64_t>(ndim), 8);
    p.caps = take(N, 4);
    p.cell_of = take(N, 4);
    p.cell_rank = take(N, 4);
    p.cell_list = take(N, 4);
    p.work = take(N, 4);
    p.nbr_cnt = take(N, 4);
    p.nbr = take(static_cast<std::uint64_t>(row_capacity) * N, 4);
    p.scan_tmp = take(2 * 4096 + 16, 4);
    if (!ok) return p;
    // The rest holds the cell grid: two arrays of C_alloc + 1 counters, each
    // starting on a 256-byte boundary. Each gets half of the remaining bytes
    // rounded down to 256, so the second array's alignment padding is covered.
    const std::size_t start = (used + 255) & ~std::size_t{255};
    if (start >= cap) return p;
    const std::size_t per_array = ((cap - start) / 2) & ~std::size_t{255};
    if (per_array < 256) return p;
    std::uint64_t cells = per_array / 4 - 1;
    const std::uint64_t cap_cells = 8 * N + 1024;
    if (cells > cap_cells) cells = cap_cells;
    if (cells > 0xFFFFFFFEull) cells = 0xFFFFFFFEull;
    p.cell_capacity = static_cast<std::uint32_t>(cells);
    p.cell_count = take(cells + 1, 4);
    p.cell_start = take(cells + 1, 4);
    p.used = used;
    p.ok = ok;
    return p;
}

}  // namespace rcpg
