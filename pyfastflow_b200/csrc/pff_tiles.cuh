// Tile decomposition shared by the label, saddle and carve kernels.
//
// The grid is cut into TILE_W x TILE_H tiles (the last row/column of tiles may be
// partial).  A cell is a tile-border cell if it sits on the first or last valid
// row or column of its tile.  For D4 receivers (every receiver is a neighbour of
// its cell, wraps included) the first cell outside a tile on any flow path is a
// tile-border cell of the next tile, which is what lets the labelling resolve
// roots over border cells only.
#pragma once
#include "pff_common.cuh"

namespace pff {

constexpr int TILE_W = 64;
constexpr int TILE_H = 32;
constexpr int TILE_CELLS = TILE_W * TILE_H;  // 2048
constexpr int TILE_THREADS = 256;
constexpr int TILE_PER_THREAD = TILE_CELLS / TILE_THREADS;  // 8

__device__ __forceinline__ bool is_tile_border(int nx, int ny, int row, int col)
{
    const int ty = row / TILE_H, tx = col / TILE_W;
    const int ly = row - ty * TILE_H, lx = col - tx * TILE_W;
    const int h = min(TILE_H, ny - ty * TILE_H), w = min(TILE_W, nx - tx * TILE_W);
    return ly == 0 || lx == 0 || ly == h - 1 || lx == w - 1;
}
__device__ __forceinline__ bool is_tile_border_i(int nx, int ny, int i)
{
    const int row = i / nx;
    return is_tile_border(nx, ny, row, i - row * nx);
}
// Border cells enumerated arithmetically: tile t = k / BORDER_SLOTS, perimeter slot
// s = k % BORDER_SLOTS (top row, bottom row, left column, right column).
constexpr int BORDER_SLOTS = 2 * TILE_W + 2 * TILE_H - 4;  // 188
__device__ __forceinline__ int border_cell(int nx, int ny, int ntx, long long k)
{
    const int t = (int)(k / BORDER_SLOTS), s = (int)(k - (long long)t * BORDER_SLOTS);
    const int tx = t % ntx, ty = t / ntx;
    const int w = min(TILE_W, nx - tx * TILE_W), h = min(TILE_H, ny - ty * TILE_H);
    int lx, ly;
    if (h == 1) {
        if (s >= w) return -1;
        lx = s; ly = 0;
    } else if (w == 1) {
        if (s >= h) return -1;
        lx = 0; ly = s;
    } else if (s < w) {
        lx = s; ly = 0;
    } else if (s < 2 * w) {
        lx = s - w; ly = h - 1;
    } else if (s < 2 * w + (h - 2)) {
        lx = 0; ly = 1 + s - 2 * w;
    } else if (s < 2 * w + 2 * (h - 2)) {
        lx = w - 1; ly = 1 + s - 2 * w - (h - 2);
    } else {
        return -1;
    }
    return (ty * TILE_H + ly) * nx + tx * TILE_W + lx;
}

__device__ __forceinline__ bool same_tile(int nx, int a, int b)
{
    const int ra = a / nx, rb = b / nx;
    return (ra / TILE_H == rb / TILE_H) && ((a - ra * nx) / TILE_W == (b - rb * nx) / TILE_W);
}

}  // namespace pff
