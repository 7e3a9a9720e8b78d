// Internal interface of the cell sort shared by sort.cu and step.cu.
#pragma once

#include <vector>

#include "common.cuh"

namespace pic {

constexpr int kSortDigitMax = 10;  // widest radix digit (bits)
constexpr int kSortPassesMax = 4;  // 32-bit keys

struct SortImpl {
    int capacity = 0, nx = 0, ny = 0, tile = 0, tiles_x = 0, tiles_y = 0, ntiles = 0;
    uint32_t dead_key = 0;
    int passes = 0, G = 0;
    int digit[kSortPassesMax] = {};  // digit width of each pass (bits)
    uint32_t *k0 = nullptr, *k1 = nullptr, *v0 = nullptr, *v1 = nullptr;
    int* cnt = nullptr;  // digit-major counts, (1 << kSortDigitMax) x G
    int* tot = nullptr;  // digit totals, 1 << kSortDigitMax
    int* n_dev = nullptr;  // [0] = n (input slots), [1] = live count
    std::vector<void*> allocs;
};

// Tiles, dead key, passes and digit widths of a sort of `capacity` slots, and
// its CTA count (at most max_ctas).
int sort_geometry(int capacity, int nx, int ny, int tile, int max_ctas, SortImpl* S);

int sorter_create(int capacity, int nx, int ny, int tile, SortImpl* S);
void sorter_free(SortImpl* S);
int sort_set_n(SortImpl& S, const int* d_n, cudaStream_t st);
int sort_passes(SortImpl& S, int* tile_start, int* count_out, const uint32_t** perm, cudaStream_t st);

// Tile-major cell key; dead particles (NaN) get dead_key.
__device__ __forceinline__ uint32_t tile_key(float gx, float gy, int ncx, int ncy, int tile, int tiles_x,
                                             uint32_t dead_key) {
    if (!is_live(gx)) return dead_key;
    int cx = int(gx), cy = int(gy);
    cx = min(cx, ncx - 1);
    cy = min(cy, ncy - 1);
    const int tx = cx / tile, ty = cy / tile;
    return uint32_t((ty * tiles_x + tx) * tile * tile + (cy - ty * tile) * tile + (cx - tx * tile));
}

}  // namespace pic
