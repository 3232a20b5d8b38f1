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
__device__ __forceinline__ bool same_tile(int nx, int a, int b)
{
    const int ra = a / nx, rb = b / nx;
    return (ra / TILE_H == rb / TILE_H) && ((a - ra * nx) / TILE_W == (b - rb * nx) / TILE_W);
}

}  // namespace pff
