// libpff lake / depression rerouting: pyfastflow/flow/lakeflow.py.
//
// Pinned semantics (the reference races in three places; all are resolved to the
// serial ascending-index result of the Taichi CPU backend with one thread):
//   - basin labels are the fixed point of pointer jumping (root+1, or 0 for an
//     outlet root), reached by any schedule on a receiver forest (:64-101);
//   - saddlesort pass 3: the saddle node is the largest qualifying cell index
//     (serial last writer, :218-219) -> atomicMax;
//   - saddlesort pass 5: the serial in-place result, computed as snapshot
//     decisions plus the one basin whose serial outcome can differ
//     (k_saddle_p5_serial_fix).
#include <cooperative_groups.h>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <cub/block/block_scan.cuh>
#include "pff_internal.h"
#include "pff_tiles.cuh"

namespace pff {

__device__ __forceinline__ long long invalid_key() { return pack_key(1e8f, 42); }  // lakeflow.py:127

__device__ __forceinline__ int warp_agg_inc(int *ctr, bool pred)
{
    const unsigned m = __ballot_sync(0xffffffffu, pred);
    if (!m) return -1;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ctr, __popc(m));
    base = __shfl_sync(0xffffffffu, base, leader);
    return pred ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

// depression_counter (:25-44) + list of the pit cells.
template <int MODE>
__global__ void k_count_pits(const int32_t *__restrict__ rec, Grid g, int *count, int *pit_list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < g.N();
    const bool pit = in && rec[i] == i && !can_leave_i<MODE>(g, i);
    const int slot = warp_agg_inc(count, pit);
    if (pit && pit_list) pit_list[slot] = i;
}

// basin_id_init (:47-61)
template <int MODE>
__global__ void k_basin_init(int32_t *bid, Grid g, const int *guard)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N() || (guard && *guard == 0)) return;
    bid[i] = can_leave_i<MODE>(g, i) ? 0 : i + 1;
}

// propagate_basin (:64-80), in place; flags[r] records any change in round r and a
// round whose predecessor changed nothing returns at once (the fixed point holds).
__global__ void __launch_bounds__(256) k_propagate(int32_t *bid, int32_t *rec_, int N, int r, int *flags)
{
    if (r > 0 && *(volatile int *)(flags + r - 1) == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int p = rec_[i];
    const int b = bid[p];
    const int pp = rec_[p];
    bool ch = false;
    if (bid[i] != b) { bid[i] = b; ch = true; }
    if (pp != p) { rec_[i] = pp; ch = true; }
    if (ch && flags[r] == 0) flags[r] = 1;
}

// ---- saddlesort (:106-281) -------------------------------------------------

// pass 2 init (:164-167), over nb = N+1 basin entries
__global__ void k_basin_arrays_init(long long *saddle, long long *outlet, int32_t *snode, uint8_t *inv, int nb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const long long iv = invalid_key();
    saddle[i] = iv;
    outlet[i] = iv;
    snode[i] = -1;
    if (inv) inv[i] = 0;
}

// pass 1 (:132-157) fused with pass 2 (:170-194): both only read the cell's own
// z' and the (stable) basin ids of its neighbours.
template <int MODE>
__global__ void __launch_bounds__(256) k_saddle_p12(const int32_t *__restrict__ bid, uint8_t *is_border, float *zp,
                                                    long long *saddle, const float *__restrict__ z, Grid g)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= g.nx || row >= g.ny) return;
    const int i = row * g.nx + col;
    const float zi = z[i];
    if (can_leave<MODE>(g, i, row, col)) { zp[i] = zi; return; }
    const int bi = bid[i];
    int js[4];
    bool border = false;
    float zn = 1e9f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = neighbour<MODE>(g, i, row, col, k);
        js[k] = j;
        if (j != -1 && bid[j] != bi) { border = true; zn = fminf(zn, z[j]); }
    }
    is_border[i] = border;
    const float zpi = border ? fmaxf(zi, zn) : 1e9f;
    zp[i] = zpi;
    if (!border) return;
    const long long iv = invalid_key();
    long long res = iv;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = js[k];
        if (j == -1) continue;
        const int bj = bid[j];
        if (bj != bi) {
            const long long c = pack_key(zpi, bj);
            res = c < res ? c : res;
        }
    }
    if (res == iv) return;
    atomicMin(saddle + bi, res);
}

// pass 3 (:199-219): saddle node = largest qualifying index (serial last writer).
template <int MODE>
__global__ void __launch_bounds__(256) k_saddle_p3(const int32_t *__restrict__ bid, const uint8_t *__restrict__ is_border,
                                                   const float *__restrict__ zp, const long long *__restrict__ saddle,
                                                   int32_t *snode, Grid g)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= g.nx || row >= g.ny) return;
    const int i = row * g.nx + col;
    if (!is_border[i]) return;
    const int bi = bid[i];
    if (bi == 0) return;
    const long long s = saddle[bi];
    const float tz = key_value(s);
    const int tb = key_index(s);
    const float zpi = zp[i];
    bool here = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = neighbour<MODE>(g, i, row, col, k);
        if (j != -1 && bid[j] == tb && zpi == tz) here = true;
    }
    if (here) atomicMax(snode + bi, i);
}

// pass 4 (:226-250): outlet = lowest foreign neighbour of the saddle node.
template <int MODE>
__global__ void k_saddle_p4(const int32_t *__restrict__ bid, const long long *__restrict__ saddle,
                            const int32_t *__restrict__ snode, long long *outlet, const float *__restrict__ z, Grid g)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < 1 || b >= g.N()) return;
    if (saddle[b] == invalid_key()) return;
    const int node = snode[b];
    if (node < 0) return;
    float tz = 1e9f;
    int r = -1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = neighbour_i<MODE>(g, node, k);
        if (j == -1) continue;
        const float zj = z[j];
        if (bid[j] != b && tz > zj) { tz = zj; r = j; }
    }
    if (r > -1) {
        const long long c = pack_key(tz, r);
        if (c < outlet[b]) outlet[b] = c;
    }
}

// pass 5 (:255-281), snapshot decisions: inv[b] = 1 if b is the larger basin of a
// 2-cycle b -> b' -> b.  Reads only the pre-pass outlet array.
__global__ void k_saddle_p5_decide(const int32_t *__restrict__ bid, const long long *__restrict__ outlet,
                                   uint8_t *inv, int N)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < 1 || b >= N) return;
    const long long o = outlet[b];
    if (o == invalid_key()) return;
    const int bd1 = bid[key_index(o)];
    if (bd1 == 0) return;
    const int ro2 = key_index(outlet[bd1]);  // invalid key -> index 42
    const int bd2 = (ro2 >= 0 && ro2 < N) ? bid[ro2] : -1;
    if (bd2 == b && bd1 < b) inv[b] = 1;
}

// Serial in-place pass 5 differs from the snapshot decisions for at most one
// basin: D = bid[42].  In serial order D reads outlet[bd1] after bd1 (< D) was
// processed; if bd1 was invalidated, the read yields the invalid key whose index
// is 42, and D is invalidated iff bid[42] == D -- true by definition of D.
__global__ void k_saddle_p5_serial_fix(const int32_t *__restrict__ bid, const long long *__restrict__ outlet,
                                       uint8_t *inv, int N)
{
    if (threadIdx.x != 0 || blockIdx.x != 0 || N <= 42) return;
    const int D = bid[42];
    if (D <= 0 || D >= N) return;
    const long long o = outlet[D];
    if (o == invalid_key()) return;
    const int bd1 = bid[key_index(o)];
    if (bd1 == 0 || bd1 >= D) return;
    if (inv[bd1]) inv[D] = 1;
}

__global__ void k_saddle_p5_apply(long long *saddle, long long *outlet, int32_t *snode, const uint8_t *__restrict__ inv,
                                  int N)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < 1 || b >= N || !inv[b]) return;
    const long long iv = invalid_key();
    outlet[b] = iv;
    saddle[b] = iv;
    snode[b] = -1;
}

// ---- carving (:308-438) -------------------------------------------------------

// init_reroute_carve second loop (:327-330): tag every saddle node.
__global__ void k_carve_tag_saddles(const int32_t *__restrict__ snode, uint8_t *tag, int N)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= N) return;
    const int s = snode[b];
    if (s != -1) tag[s] = 1;
}

// iteration_reroute_carve pass 1 (:355-359)
__global__ void k_carve_it1(const uint8_t *__restrict__ tag, uint8_t *tag_, const int32_t *__restrict__ rec,
                            int32_t *rec_, int N, int r, const int *flags)
{
    if (r > 0 && *(volatile const int *)(flags + r - 1) == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int ri = rec[i];
    if (tag[i]) tag_[ri] = 1;
    rec_[i] = ri;
}
// iteration_reroute_carve pass 2 (:362-368)
__global__ void k_carve_it2(uint8_t *tag, const uint8_t *__restrict__ tag_, int32_t *rec,
                            const int32_t *__restrict__ rec_, int N, int r, int *flags)
{
    if (r > 0 && *(volatile int *)(flags + r - 1) == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    rec[i] = rec_[rec_[i]];
    const uint8_t t = tag_[i];
    if (tag[i] != t) {
        if (flags[r] == 0) flags[r] = 1;
        tag[i] = t;
    }
}
// finalise_reroute_carve (:390-403), second loop (the first is a copy).
__global__ void k_carve_reverse(int32_t *rec, const int32_t *__restrict__ rec0, const uint8_t *__restrict__ tag, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int r = rec0[i];
    if (tag[r] && tag[i] && i != r) rec[r] = i;
}
// third loop: saddle node -> outlet node.  With dst_offset = -1 this is
// reroute_jump (:299-304): rec[b-1] = outlet node.
__global__ void k_carve_link_outlets(int32_t *rec, const int32_t *__restrict__ snode, const long long *__restrict__ outlet,
                                     int N, int jump)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= N) return;
    const long long o = outlet[b];
    if (o == invalid_key()) return;
    if (jump) rec[b - 1] = key_index(o);
    else rec[snode[b]] = key_index(o);
}


// ---- tile-resolved labels (D4 receivers) ---------------------------------------
//
// Pass T: one CTA per 64x32 tile.  Receivers are loaded into shared memory as
// tile-local pointers; pointer jumping in shared memory brings every cell to its
// tile terminal -- a root inside the tile, or the last in-tile cell of its path.
// J[i] = the root, or the receiver of the exit cell (a border cell of the next
// tile).  Border cells also seed R[i] = J[i].  The same pass lists the pits
// (interior self-receivers) and the border cells.
// Pass B: pointer jumping on R over border cells only (a few rounds).
// Pass L: bid[i] = label of root(i) = Rget(J[i]).

// R is defined at every root (R[x] = x) and every tile-border cell (its root once
// resolved) -- exactly the cells J can point at.
__device__ __forceinline__ int r_get(const int32_t *R, int nx, int ny, int x)
{
    (void)nx;
    (void)ny;
    return R[x];
}

template <int BS>
__device__ __forceinline__ void block_append(bool pred, int val, int *list, int *count)
{
    using Scan = cub::BlockScan<int, BS>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int base;
    int ex, tot;
    Scan(tmp).ExclusiveSum(pred ? 1 : 0, ex, tot);
    if (threadIdx.x == 0) base = tot ? atomicAdd(count, tot) : 0;
    __syncthreads();
    if (pred) list[base + ex] = val;
    __syncthreads();
}

// info[0] pits, info[2] set if some exit target is not a tile-border cell
// (receivers that are not D4 neighbours)
// tiles: optional list of tile ids -- recompute only those tiles; pits:
// optional (nullptr: no pit list).
template <int MODE>
__device__ void tile_terminal_one(const int32_t *__restrict__ rec, int32_t *J, int32_t *R, int *pits, int *info,
                                  const Grid &g, int tx, int ty, int *p, int *ext);

// Tile terminals of the tiles listed in tiles[0 .. *ntiles) (one block per tile,
// the grid strides over the list; the count is read on the device), or of every
// tile (tiles == NULL, a 2-D grid of tiles).
template <int MODE>
__global__ void __launch_bounds__(TILE_THREADS) k_tile_terminal(const int32_t *__restrict__ rec, int32_t *J, int32_t *R,
                                                                int *pits, int *info, Grid g, const int *tiles,
                                                                const int *ntiles)
{
    __shared__ int p[TILE_CELLS];
    __shared__ int ext[TILE_CELLS];
    if (!tiles) {
        tile_terminal_one<MODE>(rec, J, R, pits, info, g, blockIdx.x, blockIdx.y, p, ext);
        return;
    }
    const int ntx = (g.nx + TILE_W - 1) / TILE_W, n = *ntiles;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int t = tiles[k];
        tile_terminal_one<MODE>(rec, J, R, pits, info, g, t % ntx, t / ntx, p, ext);
        __syncthreads();  // p and ext are reused by the next tile
    }
}

template <int MODE>
__device__ void tile_terminal_one(const int32_t *__restrict__ rec, int32_t *J, int32_t *R, int *pits, int *info,
                                  const Grid &g, int tx, int ty, int *p, int *ext)
{
    const int nx = g.nx, ny = g.ny;
    const int col0 = tx * TILE_W, row0 = ty * TILE_H;
    const int w = min(TILE_W, nx - col0), h = min(TILE_H, ny - row0);
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; ++k) {
        const int c = threadIdx.x + k * TILE_THREADS;
        const int lx = c % TILE_W, ly = c / TILE_W;
        int pc = c, e = -2;
        if (lx < w && ly < h) {
            const int i = (row0 + ly) * nx + col0 + lx;
            const int r = rec[i];
            if (r == i) {
                e = -1;
            } else {
                int rly, rlx;
                if (r == i - 1) { rly = ly; rlx = lx - 1; }
                else if (r == i + 1) { rly = ly; rlx = lx + 1; }
                else if (r == i - nx) { rly = ly - 1; rlx = lx; }
                else if (r == i + nx) { rly = ly + 1; rlx = lx; }
                else { const int rr = r / nx; rly = rr - row0; rlx = r - rr * nx - col0; }
                if (rly >= 0 && rly < h && rlx >= 0 && rlx < w) pc = rly * TILE_W + rlx;
                else e = r;
            }
        }
        p[c] = pc;
        ext[c] = e;
    }
    __syncthreads();
    // at most ceil(log2 2048) = 11 rounds for any acyclic in-tile path.  A thread reads
    // all its cells' pointers, then all the pointers they point to, then stores: the
    // shared-memory round trips overlap (one interleaving of the same concurrent updates)
    for (int round = 0; round < 12; ++round) {
        bool ch = false;
        int q[TILE_PER_THREAD], qq[TILE_PER_THREAD];
#pragma unroll
        for (int k = 0; k < TILE_PER_THREAD; ++k) q[k] = p[threadIdx.x + k * TILE_THREADS];
#pragma unroll
        for (int k = 0; k < TILE_PER_THREAD; ++k) qq[k] = p[q[k]];
#pragma unroll
        for (int k = 0; k < TILE_PER_THREAD; ++k)
            if (qq[k] != q[k]) {
                p[threadIdx.x + k * TILE_THREADS] = qq[k];
                ch = true;
            }
        if (!__syncthreads_or(ch)) break;
    }
    bool nonlocal = false;
#pragma unroll
    for (int k = 0; k < TILE_PER_THREAD; ++k) {
        const int c = threadIdx.x + k * TILE_THREADS;
        const int lx = c % TILE_W, ly = c / TILE_W;
        bool pit = false;
        int i = -1;
        if (lx < w && ly < h) {
            i = (row0 + ly) * nx + col0 + lx;
            const int t = p[c];
            const int e = ext[t];
            const int j = (e == -1) ? (row0 + t / TILE_W) * nx + col0 + (t % TILE_W) : e;
            J[i] = j;
            if (lx == 0 || ly == 0 || lx == w - 1 || ly == h - 1 || ext[c] == -1) R[i] = j;
            if (ext[c] >= 0 && !is_tile_border_i(nx, ny, ext[c])) nonlocal = true;
            pit = pits && ext[c] == -1 && !can_leave<MODE>(g, i, row0 + ly, col0 + lx);
        }
        const unsigned m = __ballot_sync(0xffffffffu, pit);
        if (m) {
            const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(info, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (pit) pits[base + __popc(m & ((1u << lane) - 1u))] = i;
        }
    }
    if (nonlocal) info[2] = 1;
}

// Pointer jumping on R over all border cells, every round in one cooperative
// launch (grid-wide barrier between rounds); stops after a round with no change.
__global__ void __launch_bounds__(256) k_border_jump_coop(int32_t *R, int nx, int ny, int ntx, long long nslots,
                                                          int *flags)
{
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int r = 0; r < 32; ++r) {
        bool ch = false;
        for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nslots; k += stride) {
            const int e = border_cell(nx, ny, ntx, k);
            if (e < 0) continue;
            const int x = R[e];
            const int y = r_get(R, nx, ny, x);
            if (y != x) { R[e] = y; ch = true; }
        }
        if (__syncthreads_or(ch) && threadIdx.x == 0) flags[r] = 1;
        grid.sync();
        if (*(volatile int *)(flags + r) == 0) break;
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_labels_final(const int32_t *__restrict__ J, const int32_t *__restrict__ R,
                                                      int32_t *bid, Grid g, const int32_t *__restrict__ rec,
                                                      int *unresolved)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N()) return;
    const int root = r_get(R, g.nx, g.ny, J[i]);
    if (rec[root] != root) *unresolved = 1;  // a receiver cycle: labels need the general path
    bid[i] = can_leave_i<MODE>(g, root) ? 0 : root + 1;
}

// Exact quotient and remainder of n / d for 0 <= n < 2^31 and d >= 2 without the
// integer divide sequence: with m = floor(2^32 / d) or m = floor((2^32 - 1) / d) (one
// less only when d divides 2^32), q = umulhi(n, m) is floor(n / d) or one less
// (n m / 2^32 > n / d - 2 n / 2^32 > n / d - 1), and one correction of the remainder
// fixes it.
__device__ __forceinline__ void divmod_nx(int n, int d, unsigned m, int &q, int &r)
{
    q = (int)__umulhi((unsigned)n, m);
    r = n - q * d;
    if (r >= d) { ++q; r -= d; }
}

// k_labels_final on 4 cells per thread (modes 0-2, nx % 4 == 0): 16-byte loads and
// stores, the gathers of the 4 cells in flight together, and the roots' rows and
// columns without integer division.
template <int MODE>
__global__ void __launch_bounds__(256) k_labels_final4(const int32_t *__restrict__ J, const int32_t *__restrict__ R,
                                                       int32_t *bid, Grid g, const int32_t *__restrict__ rec,
                                                       int *unresolved, unsigned mnx)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (4 * q >= g.N()) return;
    const int4 j = reinterpret_cast<const int4 *>(J)[q];
    const int rt[4] = {R[j.x], R[j.y], R[j.z], R[j.w]};
    const int rr[4] = {rec[rt[0]], rec[rt[1]], rec[rt[2]], rec[rt[3]]};
    int lab[4];
    bool cyc = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        cyc |= rr[k] != rt[k];  // a receiver cycle: labels need the general path
        int row, col;
        divmod_nx(rt[k], g.nx, mnx, row, col);
        lab[k] = can_leave<MODE>(g, rt[k], row, col) ? 0 : rt[k] + 1;
    }
    reinterpret_cast<int4 *>(bid)[q] = make_int4(lab[0], lab[1], lab[2], lab[3]);
    if (cyc) *unresolved = 1;
}

// k_basin_init on 4 cells of one row per thread (modes 0-2, nx % 4 == 0)
template <int MODE>
__global__ void k_basin_init4(int32_t *bid, Grid g, const int *guard, unsigned mnx)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int i0 = 4 * q;
    if (i0 >= g.N() || (guard && *guard == 0)) return;
    int row, col;
    divmod_nx(i0, g.nx, mnx, row, col);
    int lab[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) lab[k] = can_leave<MODE>(g, i0 + k, row, col + k) ? 0 : i0 + k + 1;
    reinterpret_cast<int4 *>(bid)[q] = make_int4(lab[0], lab[1], lab[2], lab[3]);
}

// ---- list-driven saddle passes ---------------------------------------------------

// reset the basin entries of a pit list (basin = pit + 1) and entry 0
__global__ void k_basin_reset_list(long long *saddle, long long *outlet, int32_t *snode, uint8_t *inv,
                                   const int *__restrict__ pits, const int *np)
{
    const int n = *np;
    const long long iv = invalid_key();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x) {
        const int b = k < n ? pits[k] + 1 : 0;
        saddle[b] = iv;
        outlet[b] = iv;
        snode[b] = -1;
        inv[b] = 0;
    }
}

// Pass 1+2 as a column-strip stencil: each warp walks a 32-column strip down
// SAD_ROWS rows with bid and z of the rows above/at/below in registers and the
// left/right values from neighbouring lanes.  Border cells of pit basins collect
// in a per-warp shared buffer, flushed with one atomic per strip.
constexpr int SAD_ROWS = 32;
constexpr int SAD_AHEAD = 4;  // rows loaded per group (SAD_ROWS is a multiple)

// The saddle candidate of a border cell goes to atomicMin(saddle + bi, key) (pass 2).
// In the border-list pass, where most lanes hold a candidate and neighbouring list
// entries share basins, saddle_min_warp makes that one atomic per basin per warp
// (in the N-wide strip pass it cost more than it saved): the lanes holding a
// candidate group by basin (match.any), take the group's minimum key as two 32-bit
// reductions (the key's signed order is the unsigned order of key ^ 2^63: high
// words first, then the low words of the lanes that hold the minimal high word),
// and the group's first lane applies it.  The minimum over the same keys: the
// saddle is the one the per-cell atomics produce.
__device__ __forceinline__ void saddle_min_warp(long long *saddle, int bi, long long key, bool has)
{
    const unsigned act = __ballot_sync(0xffffffffu, has);
    if (!has) return;
    const unsigned peers = __match_any_sync(act, bi);
    const unsigned long long u = (unsigned long long)key ^ 0x8000000000000000ull;
    const unsigned hi = (unsigned)(u >> 32), lo = (unsigned)u;
    const unsigned mh = __reduce_min_sync(peers, hi);
    const unsigned ml = __reduce_min_sync(peers, hi == mh ? lo : 0xffffffffu);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1)
        atomicMin(saddle + bi, (long long)((((unsigned long long)mh << 32) | ml) ^ 0x8000000000000000ull));
}

// Passes 1-2 for one cell; the saddle candidate (if any) is returned in key/has.
// Returns 0 for a cell off every border, 1 for a border cell of the outlet
// basin 0, 2 for a border cell of a pit basin.
template <int MODE>
__device__ __forceinline__ int saddle_cell(int i, int row, int col, const Grid &g, int bi, float zi, const int (&jn)[4],
                                           const int (&bn)[4], const float (&zn)[4], uint8_t *is_border, float *zp,
                                           long long &key, bool &has)
{
    bool border = false;
    float zmin = 1e9f;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (jn[k] != -1 && bn[k] != bi) { border = true; zmin = fminf(zmin, zn[k]); }
    is_border[i] = border;
    const float zpi = border ? fmaxf(zi, zmin) : 1e9f;
    zp[i] = zpi;
    if (!border) return 0;
    const long long iv = invalid_key();
    long long res = iv;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (jn[k] == -1 || bn[k] == bi) continue;
        const long long c = pack_key(zpi, bn[k]);
        res = c < res ? c : res;
    }
    key = res;
    has = res != iv;
    return bi != 0 ? 2 : 1;
}

template <int MODE>
__global__ void __launch_bounds__(128) k_saddle_p12_strip(const int32_t *__restrict__ bid, uint8_t *is_border,
                                                          float *zp, long long *saddle, const float *__restrict__ z,
                                                          Grid g, int *blist, int *nblist, int *alist, int *nalist)
{
    __shared__ int buf[4][32 * SAD_ROWS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int warp = blockIdx.x * 4 + wib;
    const int nx = g.nx, ny = g.ny;
    const int nstrips = (nx + 31) >> 5;
    const int strip = warp % nstrips, band = warp / nstrips;
    const int col = (strip << 5) + lane;
    const int row0 = band * SAD_ROWS;
    if (row0 >= ny) return;
    const int row1 = min(row0 + SAD_ROWS, ny);
    const bool incol = col < nx;
    int nb = 0;  // border cells buffered by this warp
    int ba = 0, bc = 0;
    float za = 0.f, zc = 0.f;
    if (incol) {
        bc = bid[row0 * nx + col];
        zc = z[row0 * nx + col];
        if (row0 > 0) { ba = bid[(row0 - 1) * nx + col]; za = z[(row0 - 1) * nx + col]; }
    }
    // strip-edge halo columns; in periodic east-west the grid's first and last columns
    // take the wrapped column, so that they run the interior path too (no warp of the
    // edge strips waits on per-row neighbour loads)
    const bool hl = lane == 0 && incol && (col > 0 || MODE == 1);
    const bool hr = (lane == 31 || col == nx - 1) && incol && (col + 1 < nx || MODE == 1);
    const int lcol = col > 0 ? col - 1 : nx - 1, rcol = col + 1 < nx ? col + 1 : 0;
    for (int row = row0; row < row1; row += SAD_AHEAD) {
        // the rows below (and the strip-edge halo) of SAD_AHEAD rows, loaded together
        int bq[SAD_AHEAD], lq[SAD_AHEAD], rq[SAD_AHEAD];
        float zq[SAD_AHEAD], zlq[SAD_AHEAD], zrq[SAD_AHEAD];
#pragma unroll
        for (int q = 0; q < SAD_AHEAD; ++q) {
            const int rb = row + 1 + q, rc = row + q;
            const bool vb = incol && rb < ny && rb <= row1;
            bq[q] = vb ? bid[rb * nx + col] : 0;
            zq[q] = vb ? z[rb * nx + col] : 0.f;
            const bool vl = hl && rc < row1, vr = hr && rc < row1;
            lq[q] = vl ? bid[rc * nx + lcol] : 0;
            zlq[q] = vl ? z[rc * nx + lcol] : 0.f;
            rq[q] = vr ? bid[rc * nx + rcol] : 0;
            zrq[q] = vr ? z[rc * nx + rcol] : 0.f;
        }
#pragma unroll
        for (int q = 0; q < SAD_AHEAD; ++q) {
            const int rw = row + q;
            if (rw >= row1) break;
            const int i = rw * nx + col;
            const int bb = bq[q];
            const float zb = zq[q];
            int bl = __shfl_up_sync(0xffffffffu, bc, 1), br = __shfl_down_sync(0xffffffffu, bc, 1);
            float zl = __shfl_up_sync(0xffffffffu, zc, 1), zr = __shfl_down_sync(0xffffffffu, zc, 1);
            int listed = 0;  // saddle_cell's code
            long long key = 0;
            bool has = false;
            if (incol) {
                const bool interior =
                    MODE != 3 && rw > 0 && rw < ny - 1 && (MODE == 1 || (col > 0 && col < nx - 1));
                if (interior) {
                    if (hl) { bl = lq[q]; zl = zlq[q]; }
                    if (hr) { br = rq[q]; zr = zrq[q]; }
                    // interior cells of modes 0-2 never leave the domain (east-west links wrap in mode 1)
                    const int jn[4] = {i - nx, col > 0 ? i - 1 : i + nx - 1, col < nx - 1 ? i + 1 : i - nx + 1,
                                       i + nx};
                    const int bn[4] = {ba, bl, br, bb};
                    const float zn[4] = {za, zl, zr, zb};
                    listed = saddle_cell<MODE>(i, rw, col, g, bc, zc, jn, bn, zn, is_border, zp, key, has);
                } else if (can_leave<MODE>(g, i, rw, col)) {
                    zp[i] = zc;
                } else {
                    int jn[4], bn[4];
                    float zn[4];
                    neighbours4<MODE>(g, i, rw, col, jn);
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        bn[k] = jn[k] != -1 ? bid[jn[k]] : 0;
                        zn[k] = jn[k] != -1 ? z[jn[k]] : 0.f;
                    }
                    listed = saddle_cell<MODE>(i, rw, col, g, bc, zc, jn, bn, zn, is_border, zp, key, has);
                }
            }
            if (has) atomicMin(saddle + bc, key);
            // every border cell, the pit-basin ones marked by the sign bit
            const unsigned m = __ballot_sync(0xffffffffu, listed != 0);
            if (listed) buf[wib][nb + __popc(m & ((1u << lane) - 1u))] = listed == 2 ? (i | (int)0x80000000) : i;
            nb += __popc(m);
            ba = bc; bc = bb;
            za = zc; zc = zb;
        }
    }
    __syncwarp();
    int npit = 0;
    for (int k = lane; k < nb; k += 32) npit += buf[wib][k] < 0;
    npit = __reduce_add_sync(0xffffffffu, npit);
    int bp = 0, bq = 0;  // bases in blist and alist
    if (lane == 0) {
        if (npit) bp = atomicAdd(nblist, npit);
        if (alist && nb) bq = atomicAdd(nalist, nb);
    }
    bp = __shfl_sync(0xffffffffu, bp, 0);
    bq = __shfl_sync(0xffffffffu, bq, 0);
    int run = 0;
    for (int k0 = 0; k0 < nb; k0 += 32) {
        const int k = k0 + lane;
        const int v = k < nb ? buf[wib][k] : 0;
        const bool pit = k < nb && v < 0;
        const int i = v & 0x7FFFFFFF;
        if (alist && k < nb) alist[bq + k] = i;
        const unsigned m = __ballot_sync(0xffffffffu, pit);
        if (pit) blist[bp + run + __popc(m & ((1u << lane) - 1u))] = i;
        run += __popc(m);
    }
}

// Pass 1+2 with 4 columns per thread (modes 0-2, nx % 4 == 0, 16-byte aligned rows):
// a warp walks a 128-column strip down SAD4_ROWS rows with 16-byte loads of the
// labels and z, two rows of loads in flight.  A cell that cannot leave the domain
// has all four links valid in these modes (edge links wrap in the periodic ones),
// so every such cell takes the same path; edge-leaving cells only set z' = z.
// Border cells collect in a per-warp shared buffer as in k_saddle_p12_strip.
constexpr int SAD4_ROWS = 8;
template <int MODE>
__global__ void __launch_bounds__(128, 4) k_saddle_p12_strip4(const int32_t *__restrict__ bid, uint8_t *is_border,
                                                              float *zp, long long *saddle, const float *__restrict__ z,
                                                              Grid g, int *blist, int *nblist, int *alist, int *nalist)
{
    static_assert(MODE >= 0 && MODE <= 2, "custom codes take k_saddle_p12_strip");
    __shared__ int buf[4][128 * SAD4_ROWS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int warp = blockIdx.x * 4 + wib;
    const int nx = g.nx, ny = g.ny, nx4 = nx >> 2;
    const int nstrips = (nx + 127) >> 7;
    const int strip = warp % nstrips, band = warp / nstrips;
    const int c0 = (strip << 7) + 4 * lane;
    const int r0 = band * SAD4_ROWS;
    if (r0 >= ny) return;
    const int r1 = min(r0 + SAD4_ROWS, ny);
    const bool incol = c0 < nx;
    const int q0 = c0 >> 2;
    const int4 *b4 = reinterpret_cast<const int4 *>(bid);
    const float4 *z4 = reinterpret_cast<const float4 *>(z);
    // halo columns at the strip edges (wrapped in periodic east-west)
    const bool lhalo = incol && lane == 0 && (c0 > 0 || MODE == 1);
    const bool rhalo = incol && (lane == 31 || c0 + 4 == nx) && (c0 + 4 < nx || MODE == 1);
    const int lcol = c0 > 0 ? c0 - 1 : nx - 1, rcol = c0 + 4 < nx ? c0 + 4 : 0;
    // row index of the row below rw (wrapped in periodic north-south; -1: none or past the band)
    auto below = [&](int rw) -> int {
        const int rb = rw + 1;
        if (rb > r1) return -1;
        return rb < ny ? rb : (MODE == 2 ? 0 : -1);
    };
    const int4 zi4 = make_int4(0, 0, 0, 0);
    const float4 zf4 = make_float4(0.f, 0.f, 0.f, 0.f);
    int4 bc = zi4, ba = zi4;
    float4 zc = zf4, za = zf4;
    int hbl = 0, hbr = 0;
    float hzl = 0.f, hzr = 0.f;
    if (incol) {
        bc = b4[(size_t)r0 * nx4 + q0];
        zc = z4[(size_t)r0 * nx4 + q0];
        const int ra = r0 > 0 ? r0 - 1 : (MODE == 2 ? ny - 1 : -1);
        if (ra >= 0) {
            ba = b4[(size_t)ra * nx4 + q0];
            za = z4[(size_t)ra * nx4 + q0];
        }
    }
    if (lhalo) { hbl = bid[(size_t)r0 * nx + lcol]; hzl = z[(size_t)r0 * nx + lcol]; }
    if (rhalo) { hbr = bid[(size_t)r0 * nx + rcol]; hzr = z[(size_t)r0 * nx + rcol]; }
    int4 rb_[2];
    float4 rz_[2];
    int rbl[2], rbr[2];
    float rzl[2], rzr[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const int rl = below(r0 + p), rh = r0 + 1 + p;
        rb_[p] = (incol && rl >= 0) ? b4[(size_t)rl * nx4 + q0] : zi4;
        rz_[p] = (incol && rl >= 0) ? z4[(size_t)rl * nx4 + q0] : zf4;
        rbl[p] = (lhalo && rh < r1) ? bid[(size_t)rh * nx + lcol] : 0;
        rzl[p] = (lhalo && rh < r1) ? z[(size_t)rh * nx + lcol] : 0.f;
        rbr[p] = (rhalo && rh < r1) ? bid[(size_t)rh * nx + rcol] : 0;
        rzr[p] = (rhalo && rh < r1) ? z[(size_t)rh * nx + rcol] : 0.f;
    }
    int nb = 0;  // border cells buffered by this warp
    const long long iv = invalid_key();
    for (int rb0 = r0; rb0 < r1; rb0 += 2) {
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int rw = rb0 + p;
            if (rw >= r1) break;
            const int4 bb = rb_[p];
            const float4 zb = rz_[p];
            const int nbl = rbl[p], nbr = rbr[p];
            const float nzl = rzl[p], nzr = rzr[p];
            {
                const int rl = below(rw + 2), rh = rw + 3;
                rb_[p] = (incol && rl >= 0) ? b4[(size_t)rl * nx4 + q0] : zi4;
                rz_[p] = (incol && rl >= 0) ? z4[(size_t)rl * nx4 + q0] : zf4;
                rbl[p] = (lhalo && rh < r1) ? bid[(size_t)rh * nx + lcol] : 0;
                rzl[p] = (lhalo && rh < r1) ? z[(size_t)rh * nx + lcol] : 0.f;
                rbr[p] = (rhalo && rh < r1) ? bid[(size_t)rh * nx + rcol] : 0;
                rzr[p] = (rhalo && rh < r1) ? z[(size_t)rh * nx + rcol] : 0.f;
            }
            int bl = __shfl_up_sync(0xffffffffu, bc.w, 1), br = __shfl_down_sync(0xffffffffu, bc.x, 1);
            float zl = __shfl_up_sync(0xffffffffu, zc.w, 1), zr = __shfl_down_sync(0xffffffffu, zc.x, 1);
            if (lhalo) { bl = hbl; zl = hzl; }
            if (rhalo) { br = hbr; zr = hzr; }
            int listed[4] = {0, 0, 0, 0};
            if (incol) {
                const int bcv[4] = {bc.x, bc.y, bc.z, bc.w}, bav[4] = {ba.x, ba.y, ba.z, ba.w},
                          bbv[4] = {bb.x, bb.y, bb.z, bb.w};
                const float zcv[4] = {zc.x, zc.y, zc.z, zc.w}, zav[4] = {za.x, za.y, za.z, za.w},
                            zbv[4] = {zb.x, zb.y, zb.z, zb.w};
                const bool rowleave = MODE != 2 && (rw == 0 || rw == ny - 1);
                float zpo[4];
                unsigned char isb[4];
                bool wb[4];
                const int i0 = rw * nx + c0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int col = c0 + k;
                    const bool leave = rowleave || (MODE != 1 && (col == 0 || col == nx - 1));
                    const int bi = bcv[k];
                    const float zi = zcv[k];
                    // neighbours: top, left, right, bottom (all valid for a cell that cannot leave)
                    const int bn[4] = {bav[k], k > 0 ? bcv[k - 1] : bl, k < 3 ? bcv[k + 1] : br, bbv[k]};
                    const float zn[4] = {zav[k], k > 0 ? zcv[k - 1] : zl, k < 3 ? zcv[k + 1] : zr, zbv[k]};
                    bool border = false;
                    float zmin = 1e9f;
#pragma unroll
                    for (int m = 0; m < 4; ++m)
                        if (bn[m] != bi) { border = true; zmin = fminf(zmin, zn[m]); }
                    const float zpi = border ? fmaxf(zi, zmin) : 1e9f;
                    zpo[k] = leave ? zi : zpi;
                    isb[k] = border;
                    wb[k] = !leave;
                    if (!leave && border) {
                        long long res = iv;
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            if (bn[m] == bi) continue;
                            const long long cand = pack_key(zpi, bn[m]);
                            res = cand < res ? cand : res;
                        }
                        if (res != iv) atomicMin(saddle + bi, res);
                        listed[k] = bi != 0 ? 2 : 1;
                    }
                }
                reinterpret_cast<float4 *>(zp)[(size_t)rw * nx4 + q0] = make_float4(zpo[0], zpo[1], zpo[2], zpo[3]);
                if (wb[0] && wb[1] && wb[2] && wb[3]) {
                    reinterpret_cast<uchar4 *>(is_border)[(size_t)rw * nx4 + q0] = make_uchar4(isb[0], isb[1], isb[2], isb[3]);
                } else {  // a cell that can leave keeps its is_border (lakeflow.py:133-135)
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (wb[k]) is_border[i0 + k] = isb[k];
                }
            }
            // every border cell, the pit-basin ones marked by the sign bit
            const int irow = rw * nx + c0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const bool has = listed[k] != 0;
                const unsigned m = __ballot_sync(0xffffffffu, has);
                if (has)
                    buf[wib][nb + __popc(m & ((1u << lane) - 1u))] =
                        listed[k] == 2 ? ((irow + k) | (int)0x80000000) : (irow + k);
                nb += __popc(m);
            }
            ba = bc; za = zc;
            bc = bb; zc = zb;
            hbl = nbl; hzl = nzl; hbr = nbr; hzr = nzr;
        }
    }
    __syncwarp();
    int npit = 0;
    for (int k = lane; k < nb; k += 32) npit += buf[wib][k] < 0;
    npit = __reduce_add_sync(0xffffffffu, npit);
    int bp = 0, bq = 0;  // bases in blist and alist
    if (lane == 0) {
        if (npit) bp = atomicAdd(nblist, npit);
        if (alist && nb) bq = atomicAdd(nalist, nb);
    }
    bp = __shfl_sync(0xffffffffu, bp, 0);
    bq = __shfl_sync(0xffffffffu, bq, 0);
    int run = 0;
    for (int k0 = 0; k0 < nb; k0 += 32) {
        const int k = k0 + lane;
        const int v = k < nb ? buf[wib][k] : 0;
        const bool pit = k < nb && v < 0;
        const int i = v & 0x7FFFFFFF;
        if (alist && k < nb) alist[bq + k] = i;
        const unsigned m = __ballot_sync(0xffffffffu, pit);
        if (pit) blist[bp + run + __popc(m & ((1u << lane) - 1u))] = i;
        run += __popc(m);
    }
}

// Pass 1+2 of a later outer iteration over the border cells of the previous one.
// Labels change between outer iterations only by merging basins (b -> fin(b)), so
// a cell whose neighbours all shared its label still does, keeps is_border = 0
// and z' = 1e9, and contributes no saddle: only the previous border cells can
// change.  Lists the cells still on a border (all, and those of pit basins).
template <int MODE>
__global__ void __launch_bounds__(256) k_saddle_p12_border(const int32_t *__restrict__ bid, uint8_t *is_border,
                                                           float *zp, long long *saddle, const float *__restrict__ z,
                                                           Grid g, const int *__restrict__ aprev, const int *naprev,
                                                           int *anext, int *nanext, int *blist, int *nblist)
{
    const int n = *naprev;
    const int stride = gridDim.x * 256;
    const int trips = (n + stride - 1) / stride;
    const unsigned mnx = 0xffffffffu / (unsigned)g.nx;  // divmod_nx's multiplier (one division per thread)
    for (int k = 0; k < trips; ++k) {
        const int idx = k * stride + blockIdx.x * 256 + threadIdx.x;
        int code = 0, i = -1, bi = 0;
        long long key = 0;
        bool has = false;
        if (idx < n) {
            i = aprev[idx];
            int row, col;
            divmod_nx(i, g.nx, mnx, row, col);
            int jn[4], bn[4];
            float zn[4];
            neighbours4<MODE>(g, i, row, col, jn);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                bn[q] = jn[q] != -1 ? bid[jn[q]] : 0;
                zn[q] = jn[q] != -1 ? z[jn[q]] : 0.f;
            }
            // an outlet is never listed (its z' is z and it has no border status)
            bi = bid[i];
            code = saddle_cell<MODE>(i, row, col, g, bi, z[i], jn, bn, zn, is_border, zp, key, has);
        }
        saddle_min_warp(saddle, bi, key, has);
        block_append<256>(code != 0, i, anext, nanext);
        block_append<256>(code == 2, i, blist, nblist);
    }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_saddle_p3_list(const int32_t *__restrict__ bid, const float *__restrict__ zp,
                                                        const long long *__restrict__ saddle, int32_t *snode, Grid g,
                                                        const int *__restrict__ blist, const int *nblist)
{
    const int n = *nblist;
    const unsigned mnx = 0xffffffffu / (unsigned)g.nx;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = blist[k];
        const int bi = bid[i];
        const long long s = saddle[bi];
        const float tz = key_value(s);
        const int tb = key_index(s);
        const float zpi = zp[i];
        int row, col;
        divmod_nx(i, g.nx, mnx, row, col);
        bool here = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = neighbour<MODE>(g, i, row, col, q);
            if (j != -1 && bid[j] == tb && zpi == tz) here = true;
        }
        if (here) atomicMax(snode + bi, i);
    }
}

template <int MODE>
__global__ void k_saddle_p4_list(const int32_t *__restrict__ bid, const long long *__restrict__ saddle,
                                 const int32_t *__restrict__ snode, long long *outlet, const float *__restrict__ z,
                                 Grid g, const int *__restrict__ pits, const int *np)
{
    const int n = *np;
    const long long iv = invalid_key();
    const unsigned mnx = 0xffffffffu / (unsigned)g.nx;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int b = pits[k] + 1;
        if (b >= g.N() || saddle[b] == iv) continue;  // the reference's pass 4 loop stops at N-1
        const int node = snode[b];
        if (node < 0) continue;
        float tz = 1e9f;
        int r = -1;
        int row, col;
        divmod_nx(node, g.nx, mnx, row, col);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = neighbour<MODE>(g, node, row, col, q);
            if (j == -1) continue;
            const float zj = z[j];
            if (bid[j] != b && tz > zj) { tz = zj; r = j; }
        }
        if (r > -1) {
            const long long c = pack_key(tz, r);
            if (c < outlet[b]) outlet[b] = c;
        }
    }
}

__global__ void k_saddle_p5_decide_list(const int32_t *__restrict__ bid, const long long *__restrict__ outlet,
                                        uint8_t *inv, int N, const int *__restrict__ pits, const int *np)
{
    const int n = *np;
    const long long iv = invalid_key();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int b = pits[k] + 1;
        if (b >= N) continue;
        const long long o = outlet[b];
        if (o == iv) continue;
        const int bd1 = bid[key_index(o)];
        if (bd1 == 0) continue;
        const int ro2 = key_index(outlet[bd1]);
        const int bd2 = (ro2 >= 0 && ro2 < N) ? bid[ro2] : -1;
        if (bd2 == b && bd1 < b) inv[b] = 1;
    }
}

__global__ void k_saddle_p5_apply_list(long long *saddle, long long *outlet, int32_t *snode,
                                       const uint8_t *__restrict__ inv, int N, const int *__restrict__ pits,
                                       const int *np)
{
    const int n = *np;
    const long long iv = invalid_key();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int b = pits[k] + 1;
        if (b >= N || !inv[b]) continue;
        outlet[b] = iv;
        saddle[b] = iv;
        snode[b] = -1;
    }
}

// ---- carving by tile-granular path walks ------------------------------------------
//
// W1: for every basin with a saddle node, walk its path to the pit one tile at a
//     time through J (tile terminal pointers) and list the segment starts.
// W2: walk each segment inside its tile: tag the cells and reverse the links
//     (rec[next] = cell, lakeflow.py:395-397); the old receivers are read from
//     rec_, which stays unchanged until every walk is done.
// Link: rec[saddle node] = outlet node (:399-403).  Every write to rec is also
// recorded, then replayed onto rec_ so both end equal, as in the reference.
__device__ __forceinline__ void mark_tile(uint8_t *dirty, int nx, int pos)
{
    if (!dirty) return;
    const int row = pos / nx;
    dirty[(row / TILE_H) * ((nx + TILE_W - 1) / TILE_W) + (pos - row * nx) / TILE_W] = 1;
}

// Walk one path segment inside the tile of `start`: tag the cells and reverse the
// links (rec[next] = cell, :395-397), reading the old receivers from rec0.
// Returns the first cell outside the tile, or -1 if the segment ends at the pit.
__device__ __forceinline__ int walk_segment(int start, const int32_t *__restrict__ rec0, int32_t *rec, uint8_t *tag,
                                            uint8_t *tag_, int nx, uint8_t *dirty)
{
    int x = start;
    for (int step = 0; step < TILE_CELLS + 1; ++step) {
        tag[x] = 1;
        tag_[x] = 1;
        const int nxt = rec0[x];
        if (nxt == x) return -1;
        rec[nxt] = x;
        mark_tile(dirty, nx, nxt);
        if (!same_tile(nx, nxt, start)) return nxt;
        x = nxt;
    }
    return -1;
}

// Per basin with a saddle node: list the saddle node and every later segment
// start, hopping tile by tile through J (J[x] is the first cell past x's tile on
// its path, or its root).  Each warp takes 32 basins and hops them in lockstep;
// the starts collect in a per-warp shared buffer that goes out with one atomic
// when nearly full.  The paths are disjoint, so N slots suffice.
constexpr int SEG_WARPS = 4, SEG_CAP = 512;

__global__ void __launch_bounds__(32 * SEG_WARPS) k_carve_segments(const int32_t *__restrict__ snode,
                                                                   const int32_t *__restrict__ rec0,
                                                                   const int32_t *__restrict__ J,
                                                                   const int *__restrict__ pits, const int *np, int N,
                                                                   int *segs, int *nsegs, int cap, int *err)
{
    __shared__ int buf[SEG_WARPS][SEG_CAP];
    const int n = *np;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int nb = 0;  // warp-uniform
    auto flush = [&]() {
        __syncwarp();
        int base = 0;
        if (lane == 0 && nb) base = atomicAdd(nsegs, nb);
        base = __shfl_sync(0xffffffffu, base, 0);
        for (int q = lane; q < nb; q += 32) {
            if (base + q < cap) segs[base + q] = buf[wib][q];
            else *err = 1;
        }
        __syncwarp();
        nb = 0;
    };
    for (int kb = (blockIdx.x * SEG_WARPS + wib) * 32; kb < n; kb += gridDim.x * SEG_WARPS * 32) {
        const int k = kb + lane;
        int x = -1;
        if (k < n) {
            const int b = pits[k] + 1;
            if (b < N) x = snode[b];
        }
        for (int step = 0; step <= N && __any_sync(0xffffffffu, x >= 0); ++step) {
            const bool emit = x >= 0;
            const unsigned m = __ballot_sync(0xffffffffu, emit);
            if (emit) buf[wib][nb + __popc(m & ((1u << lane) - 1u))] = x;
            nb += __popc(m);
            if (nb > SEG_CAP - 32) flush();
            if (emit) x = rec0[x] == x ? -1 : J[x];
        }
    }
    flush();
}

// Walk the listed segments.  With more than WALK_BLOCK_MAX segments, one thread
// walks each in global memory (walk_segment).  Otherwise one block takes a segment:
// it loads the segment's tile with every receiver as a tile-local index (or
// ~target when the receiver lies past the tile), tags the segment's cells by
// pointer doubling (after round r every cell within 2^(r+1) - 1 steps of the
// start is tagged), then makes walk_segment's writes for the tagged cells in
// parallel: tag, tag_, rec[receiver] = cell, and the dirty tiles.
constexpr int WALK_THREADS = 256, WALK_BLOCK_MAX = 4096;

__global__ void __launch_bounds__(WALK_THREADS) k_carve_walk(const int32_t *__restrict__ rec0, int32_t *rec,
                                                             uint8_t *tag, uint8_t *tag_,
                                                             const int *__restrict__ segs, const int *nsegs, int cap,
                                                             int nx, int ny, uint8_t *dirty)
{
    __shared__ int nl[TILE_CELLS];
    __shared__ int16_t jmp[2][TILE_CELLS];
    __shared__ uint8_t on[TILE_CELLS];
    const int n = min(*nsegs, cap);
    if (n > WALK_BLOCK_MAX) {
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
            walk_segment(segs[k], rec0, rec, tag, tag_, nx, dirty);
        return;
    }
    const unsigned mnx = 0xffffffffu / (unsigned)nx;  // divmod_nx's multiplier
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
    const int s0 = segs[k];
    static_assert(TILE_W == 64, "local index = row * 64 + column");
    const int srow = s0 / nx, scol = s0 - srow * nx;
    const int ty = srow / TILE_H, tx = scol / TILE_W;
    const int r0 = ty * TILE_H, c0 = tx * TILE_W;
    const int h = min(TILE_H, ny - r0), w = min(TILE_W, nx - c0);
    const int start = ((srow - r0) << 6) | (scol - c0);
    for (int q = threadIdx.x; q < TILE_CELLS; q += WALK_THREADS) {
        const int lr = q >> 6, lc = q & 63;
        int v = q;  // cells past the grid edge: terminal, never reached
        if (lr < h && lc < w) {
            const int r = rec0[(r0 + lr) * nx + c0 + lc];
            int rr, rc;
            divmod_nx(r, nx, mnx, rr, rc);
            v = (rr / TILE_H == ty && rc / TILE_W == tx) ? (((rr - r0) << 6) | (rc - c0)) : ~r;
        }
        nl[q] = v;
        jmp[0][q] = (int16_t)((v >= 0 && v != q) ? v : -1);
        on[q] = q == start;
    }
    __syncthreads();
#pragma unroll 1
    for (int r = 0; r < 11; ++r) {  // 2^11 = TILE_CELLS
        const int16_t *jc = jmp[r & 1];
        int16_t *jn = jmp[(r & 1) ^ 1];
        for (int q = threadIdx.x; q < TILE_CELLS; q += WALK_THREADS) {
            const int j = jc[q];
            if (on[q] && j >= 0) on[j] = 1;
            jn[q] = j >= 0 ? jc[j] : (int16_t)-1;
        }
        __syncthreads();
    }
    bool local_write = false;
    for (int q = threadIdx.x; q < TILE_CELLS; q += WALK_THREADS) {
        if (!on[q]) continue;
        const int gq = (r0 + (q >> 6)) * nx + c0 + (q & 63);
        tag[gq] = 1;
        tag_[gq] = 1;
        const int v = nl[q];
        if (v == q) continue;  // the root
        if (v < 0) {
            rec[~v] = gq;  // the path leaves the tile
            mark_tile(dirty, nx, ~v);
        } else {
            rec[(r0 + (v >> 6)) * nx + c0 + (v & 63)] = gq;
            local_write = true;
        }
    }
    if (__syncthreads_or(local_write) && threadIdx.x == 0) mark_tile(dirty, nx, s0);
    }
}

__global__ void k_carve_link_list(int32_t *rec, const int32_t *__restrict__ snode, const long long *__restrict__ outlet,
                                  const int *__restrict__ pits, const int *np, int N, uint8_t *dirty, int nx)
{
    const int n = *np;
    const long long iv = invalid_key();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int b = pits[k] + 1;
        if (b >= N) continue;
        const long long o = outlet[b];
        if (o == iv) continue;
        const int s = snode[b], v = key_index(o);
        rec[s] = v;
        mark_tile(dirty, nx, s);
    }
}

// ---- next iteration's labels without relabelling from scratch ---------------------
//
// After the carve, every cell of a basin b with a valid outlet drains through its
// saddle node into basin bid[outlet node]; nothing else changes.  So the next
// labels are bid'[i] = final(bid[i]), final = the end of the chain
// b -> bid[outlet node of b] -> ..., and the next pits are the pits of the
// basins that had no valid outlet.  fin[] is indexed by basin id.
__global__ void k_relabel_init(int32_t *fin, const int32_t *__restrict__ bid, const int32_t *__restrict__ snode,
                               const long long *__restrict__ outlet, const int *__restrict__ pits, const int *np, int N,
                               int *next_pits, int *next_np, int *odd)
{
    const int n = *np;
    const long long iv = invalid_key();
    if (blockIdx.x == 0 && threadIdx.x == 0) fin[0] = 0;
    const int n32 = (n + 31) & ~31;  // whole warps iterate together (ballot below)
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n32; k += gridDim.x * blockDim.x) {
        bool keep = false;
        int p = -1;
        if (k < n) {
            p = pits[k];
            const int b = p + 1;
            const long long o = (b < N) ? outlet[b] : iv;
            if (o != iv) {
                fin[b] = bid[key_index(o)];
            } else {
                fin[b] = b;
                keep = true;
                if (b < N && snode[b] != -1) *odd = 1;  // path reversed without an outlet link
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (m) {
            const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(next_np, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (keep) next_pits[base + __popc(m & ((1u << lane) - 1u))] = p;
        }
    }
}

// fin[b] = fin[fin[b]] over the pit list.  Up to RJ_BLOCK pits one CTA does every
// round, with block barriers (its own global writes are visible to it after each);
// longer lists take the cooperative launch with grid-wide barriers.  Each kernel
// reads the count on the device and leaves the other's lists.
// Inside the reroute graph the block kernel also sets a conditional handle, so the
// cooperative launch (whose launch alone costs about 10 us) runs only for long lists.
constexpr int RJ_BLOCK = 16384;
__global__ void __launch_bounds__(1024) k_relabel_jump_block(int32_t *fin, const int *__restrict__ pits, const int *np,
                                                            cudaGraphConditionalHandle hj, int set)
{
    const int n = *np;
    if (set && threadIdx.x == 0) cudaGraphSetConditional(hj, n > RJ_BLOCK ? 1u : 0u);
    if (n > RJ_BLOCK) return;
    for (int r = 0; r < 32; ++r) {
        bool ch = false;
        for (int k = threadIdx.x; k < n; k += 1024) {
            const int b = pits[k] + 1;
            const int x = fin[b];
            const int y = fin[x];
            if (y != x) { fin[b] = y; ch = true; }
        }
        if (!__syncthreads_or(ch)) break;
    }
}
static void launch_relabel_jump_block(int32_t *fin, const int *pits, const int *np, cudaGraphConditionalHandle hj,
                                      int set, cudaStream_t st)
{
    PFF_PROBED("k_relabel_jump_block", st, k_relabel_jump_block<<<1, 1024, 0, st>>>(fin, pits, np, hj, set));
    count_launch();
}

__global__ void __launch_bounds__(256) k_relabel_jump_coop(int32_t *fin, const int *__restrict__ pits, const int *np,
                                                           int *flags)
{
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const int n = *np;
    if (n <= RJ_BLOCK) return;  // uniform over the grid: no block reaches a grid barrier
    for (int r = 0; r < 32; ++r) {
        bool ch = false;
        for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
            const int b = pits[k] + 1;
            const int x = fin[b];
            const int y = fin[x];
            if (y != x) { fin[b] = y; ch = true; }
        }
        if (__syncthreads_or(ch) && threadIdx.x == 0) flags[r] = 1;
        grid.sync();
        if (*(volatile int *)(flags + r) == 0) break;
    }
}

// four cells per thread; label 0 (outlet basins) never changes.  The same pass
// makes rec_ = rec on the carved cells (k_sync_tagged's copy, :526).
// The carve tags are consumed here: tagged cells are cleared in tag and tag_ (the
// carve tags the same cells in both), so the next carve needs no N-wide clear.
__global__ void __launch_bounds__(256) k_relabel(int32_t *bid, const int32_t *__restrict__ fin, int32_t *rec_,
                                                 const int32_t *__restrict__ rec, uint8_t *tag, uint8_t *tag_, int N,
                                                 int vec)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = 4 * q;
    if (vec && i + 3 < N) {
        int4 b = reinterpret_cast<int4 *>(bid)[q];
        const uchar4 t = reinterpret_cast<const uchar4 *>(tag)[q];
        const int4 o = b;
        if (b.x) b.x = fin[b.x];
        if (b.y) b.y = fin[b.y];
        if (b.z) b.z = fin[b.z];
        if (b.w) b.w = fin[b.w];
        if (b.x != o.x || b.y != o.y || b.z != o.z || b.w != o.w) reinterpret_cast<int4 *>(bid)[q] = b;
        if (t.x) rec_[i] = rec[i];
        if (t.y) rec_[i + 1] = rec[i + 1];
        if (t.z) rec_[i + 2] = rec[i + 2];
        if (t.w) rec_[i + 3] = rec[i + 3];
        if (t.x | t.y | t.z | t.w) {
            reinterpret_cast<uchar4 *>(tag)[q] = make_uchar4(0, 0, 0, 0);
            for (int k = i; k < i + 4; ++k) tag_[k] = 0;
        }
    } else {
        for (int k = i; k < N && k < i + 4; ++k) {
            if (bid[k]) bid[k] = fin[bid[k]];
            if (tag[k]) {
                rec_[k] = rec[k];
                tag[k] = 0;
                tag_[k] = 0;
            }
        }
    }
}

__global__ void k_dirty_list(uint8_t *dirty, int ntiles, int *list, int *count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool d = t < ntiles && dirty[t];
    if (d) dirty[t] = 0;
    const unsigned m = __ballot_sync(0xffffffffu, d);
    if (m) {
        const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(count, __popc(m));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (d) list[base + __popc(m & ((1u << lane) - 1u))] = t;
    }
}

// rec_ = rec on the carved cells: every write of the carve (reversed links and
// saddle links) is at a tagged cell, and rec == rec_ everywhere else.
__global__ void __launch_bounds__(256) k_sync_tagged(int32_t *rec_, const int32_t *__restrict__ rec,
                                                     const uint8_t *__restrict__ tag, int N, int vec,
                                                     const int *guard)
{
    if (guard && *guard == 0) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = 4 * q;
    if (vec && i + 3 < N) {
        const uchar4 t = reinterpret_cast<const uchar4 *>(tag)[q];
        if (t.x) rec_[i] = rec[i];
        if (t.y) rec_[i + 1] = rec[i + 1];
        if (t.z) rec_[i + 2] = rec[i + 2];
        if (t.w) rec_[i + 3] = rec[i + 3];
    } else {
        for (int k = i; k < N && k < i + 4; ++k)
            if (tag[k]) rec_[k] = rec[k];
    }
}

// ---- receiver cycles: the reference's serial semantics ------------------------------
//
// A carve can close a cycle of basins (b -> b' -> b'' -> b with tied saddles;
// the 2-cycle pass removes only length 2), and then the receivers hold a cycle.
// The reference resolves it in its next outer iteration through two serial
// effects, reproduced here exactly:
//   - labels: serial in-place pointer jumping (lakeflow.py:64-80) on a cycle
//     depends only on the cycle's cells, visited in ascending index; it is
//     emulated per cycle (k_cycle_emulate), every other cell takes the fixed point;
//   - reversal: several tagged cells can share a tagged receiver; the serial
//     last writer is the largest index (k_rev_claim / k_rev_apply).

// unresolved cell: its jumped pointer did not reach a true root
__global__ void k_cycle_find(const int32_t *__restrict__ rec, const int32_t *__restrict__ work, int N, int *entries,
                             int *nentries, int cap, int32_t *mark)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int r = work[i];
    if (rec[r] == r) return;
    if (atomicExch(mark + r, 1) == 0) {
        const int slot = atomicAdd(nentries, 1);
        if (slot < cap) entries[slot] = r;
    }
}

constexpr int CYC_MAX = 4096;

// One thread: walk each cycle reached by the entries, emulate the serial rounds
// on it, record the resulting label of every cycle cell in cyc_label.
template <int MODE>
__global__ void k_cycle_emulate(const int32_t *__restrict__ rec, const int *__restrict__ entries, const int *nentries,
                                int cap, int32_t *cyc_label, int32_t *done, Grid g, int rounds, int *err)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    __shared__ int cells[CYC_MAX];
    __shared__ int lrec[CYC_MAX];
    __shared__ int lbid[CYC_MAX];
    const int n = min(*nentries, cap);
    for (int e = 0; e < n; ++e) {
        int x = entries[e];
        // move onto the cycle: from any cell of a cyclic component, N steps land on it
        for (int s = 0; s < CYC_MAX && !done[x]; ++s) x = rec[x];
        if (done[x]) continue;
        // a cell reached after CYC_MAX steps lies on the cycle if the cycle is shorter
        int L = 0, y = x;
        do {
            if (L >= CYC_MAX) { *err = 1; break; }
            cells[L++] = y;
            y = rec[y];
        } while (y != x);
        if (y != x) continue;
        // ascending index order, as the serial loop visits them
        for (int a = 1; a < L; ++a) {
            int v = cells[a], b = a - 1;
            while (b >= 0 && cells[b] > v) { cells[b + 1] = cells[b]; --b; }
            cells[b + 1] = v;
        }
        for (int a = 0; a < L; ++a) {
            const int c = cells[a];
            int lo = 0, hi = L - 1, t = rec[c];
            while (lo < hi) { const int mid = (lo + hi) >> 1; if (cells[mid] < t) lo = mid + 1; else hi = mid; }
            lrec[a] = lo;
            lbid[a] = can_leave_i<MODE>(g, c) ? 0 : c + 1;
        }
        for (int r = 0; r < rounds; ++r)
            for (int a = 0; a < L; ++a) {
                lbid[a] = lbid[lrec[a]];
                lrec[a] = lrec[lrec[a]];
            }
        for (int a = 0; a < L; ++a) {
            cyc_label[cells[a]] = lbid[a];
            done[cells[a]] = 1;
            if (lbid[a] != lbid[0]) *err = 2;  // feeders' labels would depend on timing
        }
    }
}

// Unresolved cells take the label of the cycle cell their pointer ends on; all
// cells of an emulated cycle end with one label (its in-place jumping converges
// to a single self-loop), so the feeders' serial result is that label.
__global__ void k_cycle_apply(const int32_t *__restrict__ rec, const int32_t *__restrict__ work,
                              const int32_t *__restrict__ cyc_label, const int32_t *__restrict__ done, int32_t *bid, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int r = work[i];
    if (rec[r] == r) return;
    for (int s = 0; s < CYC_MAX && !done[r]; ++s) r = rec[r];
    if (done[r]) bid[i] = cyc_label[r];
}

// finalise_reroute_carve's reversal (:395-397) with the serial last writer: the
// largest tagged index claims each tagged receiver.
__global__ void k_rev_claim(const int32_t *__restrict__ rec0, const uint8_t *__restrict__ tag, int32_t *claim, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int r = rec0[i];
    if (tag[r] && tag[i] && i != r) atomicMax(claim + r, i);
}
__global__ void k_rev_apply(int32_t *rec, const int32_t *__restrict__ claim, int N)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    const int c = claim[r];
    if (c >= 0) rec[r] = c;
}

// Incremental relabel sanity.  Every acyclic chain ends at a basin that was not
// carved (no valid outlet) or at 0; a chain that ends at a carved basin came
// from a cycle (in-place jumping can collapse a cycle onto a fake fixed point, so
// convergence alone proves nothing).
__global__ void k_relabel_check(const int32_t *__restrict__ fin, const long long *__restrict__ outlet,
                                const int *__restrict__ pits, const int *np, int N, int *flag)
{
    const int n = *np;
    const long long iv = invalid_key();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int f = fin[pits[k] + 1];
        if (f != 0 && (f >= N || fin[f] != f || outlet[f] != iv)) *flag = 1;
    }
}

// ---- launchers ---------------------------------------------------------------

template <int MODE>
static void l_count_pits(const int32_t *rec, const Grid &g, int *count, int *list, cudaStream_t st)
{
    { k_count_pits<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(rec, g, count, list); count_launch(); }
}
template <int MODE>
static void l_basin_init(int32_t *bid, const Grid &g, cudaStream_t st)
{
    if (MODE != 3 && g.nx % 4 == 0 && ((uintptr_t)bid % 16) == 0) {
        const unsigned m = (unsigned)(0x100000000ull / (unsigned long long)g.nx);
        { k_basin_init4<MODE == 3 ? 0 : MODE><<<div_up(g.N() / 4, 256), 256, 0, st>>>(bid, g, nullptr, m); count_launch(); }
        return;
    }
    { k_basin_init<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(bid, g, nullptr); count_launch(); }
}
template <int MODE>
static void l_saddle(const int32_t *bid, uint8_t *isb, float *zp, long long *saddle, int32_t *snode,
                     long long *outlet, uint8_t *inv, const float *z, const Grid &g, cudaStream_t st)
{
    const int N = g.N();
    { k_basin_arrays_init<<<div_up(N + 1, 256), 256, 0, st>>>(saddle, outlet, snode, inv, N + 1); count_launch(); }
    dim3 b(32, 8), gr(div_up(g.nx, 32), div_up(g.ny, 8));
    { k_saddle_p12<MODE><<<gr, b, 0, st>>>(bid, isb, zp, saddle, z, g); count_launch(); }
    { k_saddle_p3<MODE><<<gr, b, 0, st>>>(bid, isb, zp, saddle, snode, g); count_launch(); }
    { k_saddle_p4<MODE><<<div_up(N, 256), 256, 0, st>>>(bid, saddle, snode, outlet, z, g); count_launch(); }
    { k_saddle_p5_decide<<<div_up(N, 256), 256, 0, st>>>(bid, outlet, inv, N); count_launch(); }
    { k_saddle_p5_serial_fix<<<1, 32, 0, st>>>(bid, outlet, inv, N); count_launch(); }
    { k_saddle_p5_apply<<<div_up(N, 256), 256, 0, st>>>(saddle, outlet, snode, inv, N); count_launch(); }
}

template <int MODE>
static void l_tile_terminal(const int32_t *rec, int32_t *J, int32_t *R, int *pits, int *info, const Grid &g,
                            cudaStream_t st)
{
    dim3 gr(div_up(g.nx, TILE_W), div_up(g.ny, TILE_H));
    PFF_PROBED("k_tile_terminal<grid>", st,
               k_tile_terminal<MODE><<<gr, TILE_THREADS, 0, st>>>(rec, J, R, pits, info, g, nullptr, nullptr));
    count_launch();
}
template <int MODE>
static void l_tile_terminal_list(const int32_t *rec, int32_t *J, int32_t *R, int *info, const Grid &g,
                                 const int *tiles, const int *ntiles, int grid, cudaStream_t st)
{
    // the CTAs loop over the list: no more of them than fit on the GPU at once, so that
    // none waits for a second wave with its share of the tiles
    static int resident[64];
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
        if (!resident[dev]) {
            int per = 0, nsm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tile_terminal<MODE>, TILE_THREADS, 0);
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
            resident[dev] = per > 0 && nsm > 0 ? per * nsm : -1;
        }
        if (resident[dev] > 0) grid = std::min(grid, resident[dev]);
    }
    PFF_PROBED("k_tile_terminal<list>", st,
               k_tile_terminal<MODE><<<grid, TILE_THREADS, 0, st>>>(rec, J, R, nullptr, info, g, tiles, ntiles));
    count_launch();
}
template <int MODE>
static void l_labels_final(const int32_t *J, const int32_t *R, int32_t *bid, const Grid &g, const int32_t *rec,
                           int *unresolved, cudaStream_t st)
{
    if (MODE != 3 && g.nx % 4 == 0 && ((uintptr_t)J % 16) == 0 && ((uintptr_t)bid % 16) == 0) {
        const unsigned m = (unsigned)(0x100000000ull / (unsigned long long)g.nx);
        { k_labels_final4<MODE == 3 ? 0 : MODE><<<div_up(g.N() / 4, 256), 256, 0, st>>>(J, R, bid, g, rec, unresolved, m);
          count_launch(); }
        return;
    }
    { k_labels_final<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(J, R, bid, g, rec, unresolved); count_launch(); }
}
template <int MODE>
static void l_cycle_emulate(const int32_t *rec, const int *entries, const int *n, int cap, int32_t *lab, int32_t *done,
                            const Grid &g, int rounds, int *err, cudaStream_t st)
{
    { k_cycle_emulate<MODE><<<1, 32, 0, st>>>(rec, entries, n, cap, lab, done, g, rounds, err); count_launch(); }
}
template <int MODE>
static void l_saddle_lists(const int32_t *bid, uint8_t *isb, float *zp, long long *saddle, int32_t *snode,
                           long long *outlet, uint8_t *inv, const float *z, const Grid &g, const int *pits,
                           const int *np, int *blist, int *nblist, const int *aprev, const int *naprev, int *anext,
                           int *nanext, int grid, cudaStream_t st)
{
    const int N = g.N();
    const bool vec = g.nx % 4 == 0 && ((uintptr_t)bid % 16) == 0 && ((uintptr_t)z % 16) == 0 &&
                     ((uintptr_t)zp % 16) == 0 && ((uintptr_t)isb % 4) == 0;
    if (!aprev && MODE != 3 && vec) {
        if constexpr (MODE != 3) {
            const long long warps = (long long)((g.nx + 127) / 128) * ((g.ny + SAD4_ROWS - 1) / SAD4_ROWS);
            PFF_PROBED("k_saddle_p12_strip", st,
                       k_saddle_p12_strip4<MODE><<<div_up(warps, 4), 128, 0, st>>>(bid, isb, zp, saddle, z, g, blist,
                                                                                   nblist, anext, nanext));
            count_launch();
        }
    } else if (!aprev) {
        const long long warps = (long long)((g.nx + 31) / 32) * ((g.ny + SAD_ROWS - 1) / SAD_ROWS);
        PFF_PROBED("k_saddle_p12_strip", st,
                   k_saddle_p12_strip<MODE><<<div_up(warps, 4), 128, 0, st>>>(bid, isb, zp, saddle, z, g, blist,
                                                                              nblist, anext, nanext));
        count_launch();
    } else {
        { k_saddle_p12_border<MODE><<<grid, 256, 0, st>>>(bid, isb, zp, saddle, z, g, aprev, naprev, anext, nanext,
                                                           blist, nblist); count_launch(); }
    }
    { k_saddle_p3_list<MODE><<<grid, 256, 0, st>>>(bid, zp, saddle, snode, g, blist, nblist); count_launch(); }
    { k_saddle_p4_list<MODE><<<grid, 256, 0, st>>>(bid, saddle, snode, outlet, z, g, pits, np); count_launch(); }
    { k_saddle_p5_decide_list<<<grid, 256, 0, st>>>(bid, outlet, inv, N, pits, np); count_launch(); }
    { k_saddle_p5_serial_fix<<<1, 32, 0, st>>>(bid, outlet, inv, N); count_launch(); }
    { k_saddle_p5_apply_list<<<grid, 256, 0, st>>>(saddle, outlet, snode, inv, N, pits, np); count_launch(); }
}

template <int MODE>
static void l_basin_init_if(int32_t *bid, const Grid &g, const int *guard, cudaStream_t st)
{
    if (MODE != 3 && g.nx % 4 == 0 && ((uintptr_t)bid % 16) == 0) {
        const unsigned m = (unsigned)(0x100000000ull / (unsigned long long)g.nx);
        { k_basin_init4<MODE == 3 ? 0 : MODE><<<div_up(g.N() / 4, 256), 256, 0, st>>>(bid, g, guard, m); count_launch(); }
        return;
    }
    { k_basin_init<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(bid, g, guard); count_launch(); }
}

int launch_basin_init(int32_t *bid, const Grid &g, cudaStream_t st)
{
    PFF_MODE_DISPATCH(g.mode, l_basin_init, bid, g, st);
    return check_cuda("basin_id_init");
}

static int ceil_log2(long long n)
{
    int r = 0;
    long long p = 1;
    while (p < n) { p <<= 1; ++r; }
    return r;
}

// ceil(log2 N)+1 pointer-jumping rounds on (bid, rec_work), as lakeflow.py:510-511.
int run_labels(int32_t *bid, int32_t *rec_work, const Grid &g, int *flags, cudaStream_t st)
{
    const int N = g.N();
    const int rounds = ceil_log2(N) + 1;
    PFF_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 64, st));
    for (int r = 0; r < rounds; ++r) { k_propagate<<<div_up(N, 256), 256, 0, st>>>(bid, rec_work, N, r, flags); count_launch(); }
    return check_cuda("propagate_basin");
}

int count_pits(const int32_t *rec, const Grid &g, int *dev_count, int *pit_list, int *host_count, cudaStream_t st)
{
    PFF_CUDA(cudaMemsetAsync(dev_count, 0, sizeof(int), st));
    PFF_MODE_DISPATCH(g.mode, l_count_pits, rec, g, dev_count, pit_list, st);
    PFF_TRY(check_cuda("depression_counter"));
    if (host_count) PFF_TRY(read_ints(IntReads().add(dev_count, 1), host_count, st));
    return PFF_OK;
}

}  // namespace pff

using namespace pff;

extern "C" int pff_depression_counter(const int32_t *rec, int nx, int ny, int bound_mode, const uint8_t *codes,
                                      int *count_out, void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!rec || !count_out) { set_error("pff_depression_counter: null pointer"); return PFF_ERR_ARG; }
    Grid g{nx, ny, bound_mode, codes};
    int *d = nullptr;
    PFF_CUDA(cudaMallocAsync((void **)&d, sizeof(int), S(stream)));
    int rc = count_pits(rec, g, d, nullptr, count_out, S(stream));
    cudaFreeAsync(d, S(stream));
    return rc;
}

extern "C" int pff_basin_identification(int32_t *bid, const int32_t *rec, int32_t *rec_, int nx, int ny,
                                        int bound_mode, const uint8_t *codes, void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!bid || !rec || !rec_) { set_error("pff_basin_identification: null pointer"); return PFF_ERR_ARG; }
    Grid g{nx, ny, bound_mode, codes};
    cudaStream_t st = S(stream);
    const int N = g.N();
    PFF_CUDA(cudaMemcpyAsync(rec_, rec, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    PFF_TRY(launch_basin_init(bid, g, st));
    int *flags = nullptr;
    PFF_CUDA(cudaMallocAsync((void **)&flags, sizeof(int) * 64, st));
    int rc = run_labels(bid, rec_, g, flags, st);
    cudaFreeAsync(flags, st);
    return rc;
}

extern "C" int pff_saddlesort(const int32_t *bid, uint8_t *is_border, float *z_prime, int64_t *basin_saddle,
                              int32_t *basin_saddlenode, int64_t *outlet, const float *z, int nx, int ny,
                              int bound_mode, const uint8_t *codes, void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    Grid g{nx, ny, bound_mode, codes};
    cudaStream_t st = S(stream);
    uint8_t *inv = nullptr;
    PFF_CUDA(cudaMallocAsync((void **)&inv, (size_t)g.N() + 1, st));
    PFF_MODE_DISPATCH(bound_mode, l_saddle, bid, is_border, z_prime, (long long *)basin_saddle, basin_saddlenode,
                      (long long *)outlet, inv, z, g, st);
    cudaFreeAsync(inv, st);
    return check_cuda("pff_saddlesort");
}

extern "C" size_t pff_reroute_workspace_bytes(int N)
{
    const size_t n = (size_t)N;
    return Carver::round(n + 1) * 2 + Carver::round(4 * (n + 1)) + Carver::round(4 * n) * 8 + Carver::round(8 * n) +
           Carver::round(sizeof(int) * 512) + 8192;
}

namespace pff {

struct RerouteWs {
    uint8_t *inv;
    int32_t *R, *fin;
    uint8_t *dirty;
    int *tiles;
    int *pits[2];
    int *blist, *segs;
    int *alist[2];  // every border cell of a saddlesort (parity of the outer iteration)
    int *ctr;  // [16*p + 0] pits, +2 non-D4 flag (parity p); [40] nblist, [41] nsegs, [42] nmods,
               // [43] error; [44] dirty tiles; [45] odd carve; [50 + p] alist[p] count;
               // [64..127] border-jump round flags;
               // [128..191] label round flags; [192..255] carve round flags; [256..319] relabel flags
};

static RerouteWs carve_ws(void *workspace, size_t bytes, int N)
{
    Carver cv(workspace, bytes);
    RerouteWs w;
    w.inv = cv.take<uint8_t>((size_t)N + 1);
    w.R = cv.take<int32_t>(N);
    w.fin = cv.take<int32_t>((size_t)N + 1);
    w.dirty = cv.take<uint8_t>((size_t)N);  // one byte per tile needed; N bytes bounds it
    w.tiles = cv.take<int>(N);
    w.pits[0] = cv.take<int>(N);
    w.pits[1] = cv.take<int>(N);
    w.blist = cv.take<int>(N);
    w.segs = cv.take<int>(N);
    w.alist[0] = cv.take<int>(N);
    w.alist[1] = cv.take<int>(N);
    w.ctr = cv.take<int>(512);
    return w;
}

// Tile pass over the receivers `rec`: tile terminals J into Jbuf, pit list and
// count (read back), border list.  *nonlocal_host is set if some receiver is not
// a D4 neighbour (then the tile labels do not apply).
static int tile_pass(const int32_t *rec, int32_t *Jbuf, const Grid &g, RerouteWs &w, int parity, int *npits_host,
                     int *nonlocal_host, cudaStream_t st)
{
    int *info = w.ctr + 16 * parity;
    PFF_CUDA(cudaMemsetAsync(info, 0, 4 * sizeof(int), st));
    PFF_MODE_DISPATCH(g.mode, l_tile_terminal, rec, Jbuf, w.R, w.pits[parity], info, g, st);
    int h[4];
    PFF_TRY(read_ints(IntReads().add(info, 4), h, st));
    *npits_host = h[0];
    *nonlocal_host = h[2];
    return check_cuda("tile_pass");
}

// Basin labels from a tile pass: pointer jumping over border cells, then one
// gather per cell.
static int tile_resolve(const int32_t *Jbuf, int32_t *bid, const Grid &g, RerouteWs &w, const int32_t *rec,
                        int *unresolved, cudaStream_t st)
{
    int *flags = w.ctr + 64;
    PFF_CUDA(cudaMemsetAsync(flags, 0, 64 * sizeof(int), st));
    static int coop_blocks = 0;
    if (!coop_blocks) {
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_border_jump_coop, 256, 0);
        coop_blocks = nsm * (per < 4 ? per : 4);
    }
    int nx = g.nx, ny = g.ny, ntx = div_up(g.nx, TILE_W);
    long long nslots = (long long)ntx * div_up(g.ny, TILE_H) * BORDER_SLOTS;
    int32_t *R = w.R;
    void *args[] = {&R, &nx, &ny, &ntx, &nslots, &flags};
    PFF_CUDA(cudaLaunchCooperativeKernel((void *)k_border_jump_coop, coop_blocks, 256, args, 0, st));
    count_launch();
    PFF_MODE_DISPATCH(g.mode, l_labels_final, Jbuf, w.R, bid, g, rec, unresolved, st);
    return check_cuda("tile_resolve");
}

// Labels of any receivers, with the reference's serial result on receiver
// cycles: basin_id_init, pointer-jumping rounds on work = copy of rec, then the
// cycle emulation for cells whose pointer did not reach a true root.
static int general_labels(const int32_t *rec, int32_t *work, int32_t *bid, const Grid &g, RerouteWs &w, int *err,
                          cudaStream_t st)
{
    const int N = g.N();
    PFF_TRY(launch_basin_init(bid, g, st));
    PFF_CUDA(cudaMemcpyAsync(work, rec, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    PFF_TRY(run_labels(bid, work, g, w.ctr + 128, st));
    int *nentries = w.ctr + 46;
    PFF_CUDA(cudaMemsetAsync(nentries, 0, sizeof(int), st));
    PFF_CUDA(cudaMemsetAsync(w.segs, 0, sizeof(int) * (size_t)N, st));   // mark
    PFF_CUDA(cudaMemsetAsync(w.blist, 0, sizeof(int) * (size_t)N, st));  // done
    { k_cycle_find<<<div_up(N, 256), 256, 0, st>>>(rec, work, N, w.tiles, nentries, N, w.segs); count_launch(); }
    PFF_MODE_DISPATCH(g.mode, l_cycle_emulate, rec, w.tiles, nentries, N, w.fin, w.blist, g, ceil_log2(N) + 1, err,
                      st);
    { k_cycle_apply<<<div_up(N, 256), 256, 0, st>>>(rec, work, w.fin, w.blist, bid, N); count_launch(); }
    return check_cuda("general_labels");
}

}  // namespace pff

namespace pff {
// ---- the outer loop of reroute_flow driven on the device (carve rerouting) -------------
// The host-driven loop reads pit counts and flags once per outer iteration to
// decide whether to go on.  Here the decisions are made by one-thread kernels
// that set CUDA-graph conditional handles, so a whole call is one graph launch:
//
//   prologue: rec_ = rec, counters zeroed, tile terminals + pit list
//   plan0 (IF pits and D4 receivers):
//     labels by border pointer jumping; plan1 (IF no receiver cycle):
//       iteration 0 (strip saddle pass, carve, relabel preparation); decide
//       WHILE (go on): iteration (parity 1); decide; IF (go on): iteration (parity 0); decide
//   basin_id_init (:537) when the loop ended normally
//
// Two iterations per WHILE body keep every kernel argument fixed (the list
// buffers alternate with the iteration's parity).  decide mirrors the host loop's
// tests in its order (:500, :512-514 and the carve checks) and stops the loop
// after at most outer <= 32 iterations.  The rare cases that need the
// reference's N-wide steps (non-D4 receivers, receiver cycles) stop the graph in
// a recorded state; the host then runs those steps from there.
//
// ctl = w.ctr + RR_CTL: [0] iteration, [1] outer, [2] n_outer, [3] state,
// [4] sync_tagged needed, [5] basin_init needed, [6] plan0 passed, [7] plan1
// passed, [8] iterations run.
enum { RR_RUN = 0, RR_NOPITS = 1, RR_DONE = 2, RR_GENERAL = 3, RR_RESUME = 4, RR_WALKERR = 5, RR_BOUND = 6 };
constexpr int RR_CTL = 400;

__device__ __forceinline__ int d_ceil_log2(long long n)
{
    int r = 0;
    long long p = 1;
    while (p < n) { p <<= 1; ++r; }
    return r;
}

__global__ void k_rr_plan0(int *ctl, const int *info, cudaGraphConditionalHandle ha)
{
    if (threadIdx.x) return;
    const int npits = info[0], nonlocal = info[2];
    for (int k = 0; k < 9; ++k) ctl[k] = 0;
    int go = 0;
    if (npits == 0) ctl[3] = RR_NOPITS;                 // :496-497
    else {
        ctl[1] = d_ceil_log2(npits) + 1;                // :500
        if (nonlocal) ctl[3] = RR_GENERAL;
        else { ctl[3] = RR_RUN; go = 1; }
    }
    ctl[6] = go;
    cudaGraphSetConditional(ha, go);
}

__global__ void k_rr_plan1(int *ctl, const int *unresolved, cudaGraphConditionalHandle hb)
{
    if (threadIdx.x) return;
    const int go = *unresolved ? 0 : 1;
    if (!go) ctl[3] = RR_GENERAL;  // the input receivers hold a cycle
    ctl[7] = go;
    cudaGraphSetConditional(hb, go);
}

__global__ void k_rr_decide(int *ctl, const int *ctr, const int *np_next, cudaGraphConditionalHandle hc,
                            cudaGraphConditionalHandle hm, int set_hm)
{
    if (threadIdx.x) return;
    const int it = ctl[0], outer = ctl[1];
    int n_outer = ctl[2] + 1;
    const int walk_err = ctr[43], odd = ctr[45], cycle = ctr[49], nd_next = *np_next;
    int state = RR_RUN;
    if (walk_err) state = RR_WALKERR;
    else if (odd) state = RR_RESUME;              // a reversed path without an outlet link
    else if (it + 1 >= outer) state = RR_DONE;    // :500
    else if (cycle) state = RR_RESUME;            // the carve closed a receiver cycle
    else if (nd_next == 0) { ++n_outer; state = RR_DONE; }  // the next count is 0 (:512-514)
    else if (it + 1 >= 64) state = RR_BOUND;
    ctl[2] = n_outer;
    ctl[3] = state;
    ctl[4] = state != RR_RUN;                     // rec_ = rec on the carved cells before stopping
    ctl[5] = state == RR_DONE || state == RR_WALKERR;
    ctl[8] += 1;
    if (state == RR_RUN) ctl[0] = it + 1;
    cudaGraphSetConditional(hc, state == RR_RUN);
    if (set_hm) cudaGraphSetConditional(hm, state == RR_RUN);
}

struct RRBufs {
    int32_t *bid, *rec, *rec_, *rec__;
    const float *z;
    float *zp;
    uint8_t *isb;
    long long *out, *sad;
    int32_t *snode;
    uint8_t *tag, *tag_;
    Grid g;
    RerouteWs w;
};

static int coop_blocks_for(const void *fn)
{
    int dev = 0, nsm = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 256, 0);
    return nsm * (per < 4 ? per : 4);
}

// One fast outer iteration with list parity par, enqueued on s (captured).  first:
// iteration 0 (labels come from the prologue); otherwise it starts with the basin
// relabelling and the dirty tiles' terminals that the previous iteration's
// decision asked for.
static int rr_cond(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaGraph_t *body);
static int rr_handle(cudaStream_t s, cudaGraphConditionalHandle *h);

// One outer iteration, captured on s (inside the reroute graph); aux captures the
// body of the conditional cooperative relabel launch.
static int rr_iteration(const RRBufs &A, int par, bool first, cudaStream_t s, cudaStream_t aux)
{
    const Grid &g = A.g;
    const RerouteWs &w = A.w;
    const int N = g.N(), nx = g.nx, B = 256;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * 8;
    const int ntx = div_up(nx, TILE_W), ntiles = ntx * div_up(g.ny, TILE_H);
    int *np = w.ctr + 16 * par, *np_next = w.ctr + 16 * (par ^ 1);
    if (!first) {
        { k_relabel<<<div_up(div_up(N, 4), B), B, 0, s>>>(A.bid, w.fin, A.rec_, A.rec, A.tag, A.tag_, N,
                                                         ((uintptr_t)A.bid & 15) == 0 && ((uintptr_t)A.tag & 3) == 0); count_launch(); }
        PFF_MODE_DISPATCH(g.mode, l_tile_terminal_list, A.rec_, A.rec__, w.R, np_next, g, w.tiles, w.ctr + 44,
                          std::min(ntiles, grid), s);
        { k_basin_reset_list<<<grid, B, 0, s>>>(A.sad, A.out, A.snode, w.inv, w.pits[par ^ 1], np_next); count_launch(); }
    } else {
        { k_basin_arrays_init<<<div_up(N + 1, B), B, 0, s>>>(A.sad, A.out, A.snode, w.inv, N + 1); count_launch(); }
    }
    PFF_CUDA(cudaMemsetAsync(w.ctr + 40, 0, 6 * sizeof(int), s));
    PFF_CUDA(cudaMemsetAsync(w.ctr + 50 + par, 0, sizeof(int), s));
    PFF_MODE_DISPATCH(g.mode, l_saddle_lists, A.bid, A.isb, A.zp, A.sad, A.snode, A.out, w.inv, A.z, g, w.pits[par],
                      np, w.blist, w.ctr + 40, first ? nullptr : w.alist[par ^ 1], w.ctr + 50 + (par ^ 1),
                      w.alist[par], w.ctr + 50 + par, grid, s);
    if (first) {  // later iterations: k_relabel cleared the previous carve's tags
        PFF_CUDA(cudaMemsetAsync(A.tag, 0, (size_t)N, s));
        PFF_CUDA(cudaMemsetAsync(A.tag_, 0, (size_t)N, s));
    }
    { k_carve_segments<<<nsm * 4, 32 * SEG_WARPS, 0, s>>>(A.snode, A.rec_, A.rec__, w.pits[par], np, N, w.segs,
                                                           w.ctr + 41, N, w.ctr + 43); count_launch(); }
    { k_carve_walk<<<nsm * 4, WALK_THREADS, 0, s>>>(A.rec_, A.rec, A.tag, A.tag_, w.segs, w.ctr + 41, N, nx, g.ny,
                                                     w.dirty); count_launch(); }
    { k_carve_link_list<<<grid, B, 0, s>>>(A.rec, A.snode, A.out, w.pits[par], np, N, w.dirty, nx); count_launch(); }
    PFF_CUDA(cudaMemsetAsync(np_next, 0, 4 * sizeof(int), s));
    { k_relabel_init<<<grid, B, 0, s>>>(w.fin, A.bid, A.snode, A.out, w.pits[par], np, N, w.pits[par ^ 1], np_next,
                                        w.ctr + 45); count_launch(); }
    { k_dirty_list<<<div_up(ntiles, B), B, 0, s>>>(w.dirty, ntiles, w.tiles, w.ctr + 44); count_launch(); }
    int *flags = w.ctr + 256;
    PFF_CUDA(cudaMemsetAsync(flags, 0, 64 * sizeof(int), s));
    static int coop_relabel = 0;
    if (!coop_relabel) coop_relabel = coop_blocks_for((const void *)k_relabel_jump_coop);
    int *plist = w.pits[par];
    int32_t *fin = w.fin;
    cudaGraphConditionalHandle hj;
    PFF_TRY(rr_handle(s, &hj));
    launch_relabel_jump_block(fin, plist, np, hj, 1, s);
    cudaGraph_t jbody = nullptr;
    PFF_TRY(rr_cond(s, hj, cudaGraphCondTypeIf, &jbody));
    PFF_CUDA(cudaStreamBeginCaptureToGraph(aux, jbody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    void *args[] = {&fin, &plist, &np, &flags};
    // not counted: the graph's launch tally counts it once per replay, and it runs
    // only for pit lists longer than RJ_BLOCK
    const cudaError_t le = cudaLaunchCooperativeKernel((void *)k_relabel_jump_coop, coop_relabel, 256, args, 0, aux);
    cudaGraph_t captured = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(aux, &captured);
    PFF_CUDA(le);
    PFF_CUDA(ee);
    PFF_CUDA(cudaMemsetAsync(w.ctr + 49, 0, sizeof(int), s));
    { k_relabel_check<<<grid, B, 0, s>>>(w.fin, A.out, w.pits[par], np, N, w.ctr + 49); count_launch(); }
    return check_cuda("reroute iteration");
}

// streams used to capture the graph's nested bodies (one per nesting depth)
static cudaStream_t rr_capture_stream(int dev, int depth)
{
    static cudaStream_t streams[64][10];
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!streams[dev][depth]) cudaStreamCreateWithFlags(&streams[dev][depth], cudaStreamNonBlocking);
    return streams[dev][depth];
}

// a conditional node after the current capture frontier of s; its body graph is returned
static int rr_cond(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, cudaGraph_t *body)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t gr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    PFF_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &gr, &deps, &nd));
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    PFF_CUDA(cudaGraphAddNode(&node, gr, deps, nd, &p));
    *body = p.conditional.phGraph_out[0];
    PFF_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return PFF_OK;
}

static int rr_handle(cudaStream_t s, cudaGraphConditionalHandle *h)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t gr;
    PFF_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &gr, nullptr, nullptr));
    PFF_CUDA(cudaGraphConditionalHandleCreate(h, gr, 0, cudaGraphCondAssignDefault));
    return PFF_OK;
}

struct RRKernelCounts {
    long long pro, a, b0, it2;  // kernels in the prologue, body A, iteration 0, a parity-1 iteration + decide
    long long tail;             // the state copy at the end (graphs built for pff_reroute_flow_async)
};

// the final state words (RR_CTL .. +8) into the caller's device buffer
// (out may be pinned host memory, written through its unified address)
__global__ void k_rr_ctl_copy(const int *ctl, int *out)
{
    if (threadIdx.x < 9) ((volatile int *)out)[threadIdx.x] = ctl[threadIdx.x];
}

// Capture the whole graph.  Every capture begun here is ended on every path.
static int rr_capture(const RRBufs &A, int dev, cudaGraph_t G, RRKernelCounts *kc, int *ctl_out)
{
    const Grid &g = A.g;
    const RerouteWs &w = A.w;
    const int N = g.N();
    const size_t nb4 = sizeof(int32_t) * (size_t)N;
    const int ntx = div_up(g.nx, TILE_W), ntiles = ntx * div_up(g.ny, TILE_H);
    int *ctl = w.ctr + RR_CTL;
    cudaStream_t s[5];
    for (int d = 0; d < 5; ++d) {
        s[d] = rr_capture_stream(dev, d);
        if (!s[d]) { set_error("reroute graph: no capture stream"); return PFF_ERR_CUDA; }
    }
    int depth = 0, rc = PFF_OK;
    cudaGraph_t body[5] = {G, nullptr, nullptr, nullptr, nullptr};
    auto begin = [&](int d) -> int {
        PFF_CUDA(cudaStreamBeginCaptureToGraph(s[d], body[d], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        depth = d + 1;
        return PFF_OK;
    };
    long long l0 = g_launches.load();
    do {
        if ((rc = begin(0))) break;
        // prologue (:491)
        if (cudaMemcpyAsync(A.rec_, A.rec, nb4, cudaMemcpyDeviceToDevice, s[0]) != cudaSuccess ||
            cudaMemsetAsync(w.ctr, 0, 512 * sizeof(int), s[0]) != cudaSuccess ||
            cudaMemsetAsync(w.dirty, 0, (size_t)ntiles, s[0]) != cudaSuccess) { rc = check_cuda("reroute graph"); break; }
        PFF_MODE_DISPATCH(g.mode, l_tile_terminal, A.rec_, A.rec__, w.R, w.pits[0], w.ctr, g, s[0]);
        cudaGraphConditionalHandle ha, hb, hc, hm;
        if ((rc = rr_handle(s[0], &ha))) break;
        { k_rr_plan0<<<1, 32, 0, s[0]>>>(ctl, w.ctr, ha); count_launch(); }
        kc->pro = g_launches.load() - l0;
        l0 = g_launches.load();
        if ((rc = rr_cond(s[0], ha, cudaGraphCondTypeIf, &body[1]))) break;
        if ((rc = begin(1))) break;
        // labels: pointer jumping over border cells, one gather per cell
        if (cudaMemsetAsync(w.ctr + 64, 0, 64 * sizeof(int), s[1]) != cudaSuccess ||
            cudaMemsetAsync(w.ctr + 48, 0, sizeof(int), s[1]) != cudaSuccess) { rc = check_cuda("reroute graph"); break; }
        {
            static int coop_border = 0;
            if (!coop_border) coop_border = coop_blocks_for((const void *)k_border_jump_coop);
            int nx = g.nx, ny = g.ny, tx = ntx;
            long long nslots = (long long)ntx * div_up(g.ny, TILE_H) * BORDER_SLOTS;
            int32_t *R = w.R;
            int *flags = w.ctr + 64;
            void *args[] = {&R, &nx, &ny, &tx, &nslots, &flags};
            if (cudaLaunchCooperativeKernel((void *)k_border_jump_coop, coop_border, 256, args, 0, s[1]) != cudaSuccess) {
                rc = check_cuda("reroute graph: cooperative launch");
                break;
            }
            count_launch();
        }
        PFF_MODE_DISPATCH(g.mode, l_labels_final, A.rec__, w.R, A.bid, g, A.rec_, w.ctr + 48, s[1]);
        if ((rc = rr_handle(s[1], &hb))) break;
        { k_rr_plan1<<<1, 32, 0, s[1]>>>(ctl, w.ctr + 48, hb); count_launch(); }
        kc->a = g_launches.load() - l0;
        l0 = g_launches.load();
        if ((rc = rr_cond(s[1], hb, cudaGraphCondTypeIf, &body[2]))) break;
        if ((rc = begin(2))) break;
        if ((rc = rr_iteration(A, 0, true, s[2], rr_capture_stream(dev, 7)))) break;
        if ((rc = rr_handle(s[2], &hc))) break;
        { k_rr_decide<<<1, 32, 0, s[2]>>>(ctl, w.ctr, w.ctr + 16, hc, hc, 0); count_launch(); }
        { k_sync_tagged<<<div_up(div_up(N, 4), 256), 256, 0, s[2]>>>(A.rec_, A.rec, A.tag, N,
                                                                   ((uintptr_t)A.tag & 3) == 0, ctl + 4); count_launch(); }
        kc->b0 = g_launches.load() - l0;
        l0 = g_launches.load();
        if ((rc = rr_cond(s[2], hc, cudaGraphCondTypeWhile, &body[3]))) break;
        if ((rc = begin(3))) break;
        if ((rc = rr_iteration(A, 1, false, s[3], rr_capture_stream(dev, 8)))) break;
        if ((rc = rr_handle(s[3], &hm))) break;
        { k_rr_decide<<<1, 32, 0, s[3]>>>(ctl, w.ctr, w.ctr, hc, hm, 1); count_launch(); }
        { k_sync_tagged<<<div_up(div_up(N, 4), 256), 256, 0, s[3]>>>(A.rec_, A.rec, A.tag, N,
                                                                   ((uintptr_t)A.tag & 3) == 0, ctl + 4); count_launch(); }
        kc->it2 = g_launches.load() - l0;
        if ((rc = rr_cond(s[3], hm, cudaGraphCondTypeIf, &body[4]))) break;
        if ((rc = begin(4))) break;
        if ((rc = rr_iteration(A, 0, false, s[4], rr_capture_stream(dev, 9)))) break;
        { k_rr_decide<<<1, 32, 0, s[4]>>>(ctl, w.ctr, w.ctr + 16, hc, hc, 0); count_launch(); }
        { k_sync_tagged<<<div_up(div_up(N, 4), 256), 256, 0, s[4]>>>(A.rec_, A.rec, A.tag, N,
                                                                   ((uintptr_t)A.tag & 3) == 0, ctl + 4); count_launch(); }
        // close the bodies, innermost first; then basin_id_init on the top level
        for (int d = 4; d >= 1; --d) {
            cudaGraph_t out_g;
            if (cudaStreamEndCapture(s[d], &out_g) != cudaSuccess) { rc = check_cuda("reroute graph: end capture"); break; }
            depth = d;
        }
        if (rc) break;
        PFF_MODE_DISPATCH(g.mode, l_basin_init_if, A.bid, g, ctl + 5, s[0]);
        if (ctl_out) {
            l0 = g_launches.load();
            { k_rr_ctl_copy<<<1, 32, 0, s[0]>>>(ctl, ctl_out); count_launch(); }
            kc->tail = g_launches.load() - l0;
        }
    } while (0);
    // end every capture still open (innermost first)
    for (int d = depth - 1; d >= 0; --d) {
        cudaGraph_t out_g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s[d], &out_g);
        if (e != cudaSuccess && rc == PFF_OK) {
            set_error("reroute graph: end capture: %s", cudaGetErrorString(e));
            rc = PFF_ERR_CUDA;
        }
    }
    cudaGetLastError();
    return rc;
}

// every pointer and size the graph bakes in, as plain 64-bit words (no padding)
struct RRKey {
    unsigned long long v[32];
    int n = 0;
    void add(unsigned long long x) { v[n++] = x; }
    void add(const void *p) { v[n++] = (unsigned long long)(uintptr_t)p; }
    bool operator==(const RRKey &o) const { return n == o.n && std::memcmp(v, o.v, sizeof(v[0]) * n) == 0; }
};
struct RREntry {
    RRKey key;
    cudaGraphExec_t exec = nullptr;
    RRKernelCounts kc{};
};

// Whether pff_reroute_flow runs its outer loop from a device-driven graph (default)
// or from the host loop; PFF_REROUTE_NO_GRAPH in the environment turns the default
// off, pff_reroute_use_graphs changes it at run time.
static std::atomic<int> g_rr_graphs{-1};
static bool rr_graphs_on()
{
    int v = g_rr_graphs.load();
    if (v < 0) {
        int fresh = getenv("PFF_REROUTE_NO_GRAPH") != nullptr ? 0 : 1;
        if (!g_rr_graphs.compare_exchange_strong(v, fresh)) return g_rr_graphs.load() != 0;
        v = fresh;
    }
    return v != 0;
}

// Launch the device-driven loop for these buffers (a graph built and kept on the
// first call with them), then read its final state (one synchronisation).
// Returns PFF_ERR_UNSUPPORTED when graphs cannot be built here.
// Kernels one launch of a graph ran, from its final state words c[0..8].
static long long rr_tally(const RRKernelCounts &kc, const int *c)
{
    long long nk = kc.pro + kc.tail;  // prologue, body A, iteration 0, then the iterations of the WHILE
    if (c[6]) nk += kc.a;
    if (c[7] && c[8] > 0) nk += kc.b0 + (long long)(c[8] - 1) * kc.it2;
    return nk + (c[5] ? 1 : 0);  // + basin_id_init
}

// ctl_out: NULL, or a device buffer of 9 ints that the graph's last node fills with its
// final state (a separate graph variant).  launch_only: return after the launch (the
// caller reads the state later); kc_out receives the graph's kernel counts.
static int reroute_graph(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z, float *z_prime,
                         uint8_t *is_border, long long *out, long long *sad, int32_t *snode, uint8_t *tag,
                         uint8_t *tag_, const Grid &g, RerouteWs &w, void *workspace, size_t workspace_bytes,
                         int *state, int *it, int *outer, int *n_outer, cudaStream_t st, int *ctl_out = nullptr,
                         bool launch_only = false, RRKernelCounts *kc_out = nullptr)
{
    static std::mutex mu;
    static RREntry cache[8];
    static int next = 0;
    if (!rr_graphs_on()) return PFF_ERR_UNSUPPORTED;
    (void)workspace;
    (void)workspace_bytes;
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return PFF_ERR_UNSUPPORTED;
    const RRBufs bufs{bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, snode, tag, tag_, g, w};
    RRKey key;
    for (const void *p : {(const void *)bid, (const void *)rec, (const void *)rec_, (const void *)rec__,
                          (const void *)z, (const void *)z_prime, (const void *)is_border, (const void *)out,
                          (const void *)sad, (const void *)snode, (const void *)tag, (const void *)tag_,
                          (const void *)g.codes, (const void *)w.inv, (const void *)w.ctr, (const void *)ctl_out})
        key.add(p);
    key.add((unsigned long long)g.nx);
    key.add((unsigned long long)g.ny);
    key.add((unsigned long long)g.mode);
    key.add((unsigned long long)dev);
    cudaGraphExec_t exec = nullptr;
    RRKernelCounts kc{};
    {
        std::lock_guard<std::mutex> lk(mu);
        for (auto &e : cache)
            if (e.exec && e.key == key) { exec = e.exec; kc = e.kc; }
        if (!exec) {
            cudaGraph_t G = nullptr;
            PFF_CUDA(cudaGraphCreate(&G, 0));
            const long long l0 = g_launches.load();
            int rc = rr_capture(bufs, dev, G, &kc, ctl_out);
            g_launches.store(l0);  // captured, not launched: replays are counted below
            if (rc == PFF_OK && cudaGraphInstantiate(&exec, G, 0) != cudaSuccess) {
                set_error("reroute graph: instantiate: %s", cudaGetErrorString(cudaGetLastError()));
                exec = nullptr;
                rc = PFF_ERR_UNSUPPORTED;
            }
            cudaGraphDestroy(G);
            if (rc != PFF_OK) {
                cudaGetLastError();
                return PFF_ERR_UNSUPPORTED;
            }
            RREntry &e = cache[next];
            next = (next + 1) % 8;
            if (e.exec) cudaGraphExecDestroy(e.exec);
            e.key = key;
            e.exec = exec;
            e.kc = kc;
        }
    }
    PFF_CUDA(cudaGraphLaunch(exec, st));
    if (kc_out) *kc_out = kc;
    if (launch_only) return check_cuda("reroute graph launch");
    int c[9];
    PFF_TRY(read_ints(IntReads().add(w.ctr + RR_CTL, 9), c, st));
    *it = c[0];
    *outer = c[1];
    *n_outer = c[2];
    *state = c[3];
    g_launches.fetch_add(rr_tally(kc, c));
    return check_cuda("reroute graph launch");
}

// The outer loop of reroute_flow driven from the host, from iteration it_start
// (0: from the start; else resuming after a device-driven iteration, in general
// mode, with outer and n_outer as they were).  Ends with basin_id_init (:537) and
// the error checks.
static int reroute_host_loop(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                             float *z_prime, uint8_t *is_border, long long *out, long long *sad,
                             int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int carve, const Grid &g,
                             RerouteWs &w, int it_start, int outer, bool general, int n_outer, int *n_outer_out,
                             cudaStream_t st)
{
    const int N = g.N(), nx = g.nx, bound_mode = g.mode;
    const size_t nb4 = sizeof(int32_t) * (size_t)N;
    const int B = 256, nbk = div_up(N, B);
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * 8;
    const int ntx = div_up(nx, TILE_W), ntiles = ntx * div_up(g.ny, TILE_H);
    // Fast mode (carve, D4 receivers, no receiver cycle): tile labels in the first
    // iteration, basin relabelling and dirty-tile terminals afterwards, list-driven
    // saddle passes, tile-walk carving.  General mode (jump rerouting, non-D4
    // receivers, or once a receiver cycle appears): the reference's own steps with
    // its serial semantics, N-wide.
    bool incremental = false;
    int nd_next = 0;
    int *cyc_err = w.ctr + 47;
    static const bool trace = getenv("PFF_TRACE_REROUTE") != nullptr;  // diagnostic trace on stderr
    for (int it = it_start;; ++it) {
        if (it > 0 && it >= outer) break;  // :500
        const int par = it & 1;
        int *np = w.ctr + 16 * par;
        int nd_bis = 0;
        if (incremental && !general) {
            nd_bis = nd_next;  // pits left after the previous carve; bid already relabelled
        } else if (!general && it == 0) {
            int nonlocal = 0;
            PFF_TRY(tile_pass(rec_, rec__, g, w, par, &nd_bis, &nonlocal, st));  // :493, :501
            if (nonlocal) general = true;
        } else {
            PFF_CUDA(cudaMemsetAsync(np, 0, 4 * sizeof(int), st));
            PFF_MODE_DISPATCH(g.mode, l_count_pits, rec_, g, np, w.pits[par], st);  // :501
            PFF_TRY(read_ints(IntReads().add(np, 1), &nd_bis, st));
        }
        if (it == 0) {
            if (nd_bis == 0) return check_cuda("pff_reroute_flow");  // :496-497, bid untouched
            outer = ceil_log2(nd_bis) + 1;                            // :500
        }
        // basin labels: basin_id_init + propagate_basin on rec__ = rec_ (:507-511)
        if (!general && !incremental) {
            int *unres = w.ctr + 48;
            PFF_CUDA(cudaMemsetAsync(unres, 0, sizeof(int), st));
            PFF_TRY(tile_resolve(rec__, bid, g, w, rec_, unres, st));
            int u = 0;
            PFF_TRY(read_ints(IntReads().add(unres, 1), &u, st));
            if (u) general = true;  // the input receivers hold a cycle
        }
        if (general) PFF_TRY(general_labels(rec_, rec__, bid, g, w, cyc_err, st));
        if (trace) fprintf(stderr, "[pff reroute] it %d outer %d pits %d general %d incremental %d\n", it, outer, nd_bis,
                           (int)general, (int)incremental);
        ++n_outer;
        if (nd_bis == 0) break;  // :512-514
        // ---- saddlesort (:520) ----
        if (general) {
            // every basin id, as the reference loops (cycle basins are not pits)
            PFF_MODE_DISPATCH(bound_mode, l_saddle, bid, is_border, z_prime, sad, basin_saddlenode, out, w.inv, z, g, st);
        } else {
            if (it == 0) {
                { k_basin_arrays_init<<<div_up(N + 1, B), B, 0, st>>>(sad, out, basin_saddlenode, w.inv, N + 1); count_launch(); }
            } else {
                // the previous saddlesort wrote only the entries of its pits (a superset of the current ones) and 0
                { k_basin_reset_list<<<grid, B, 0, st>>>(sad, out, basin_saddlenode, w.inv, w.pits[par ^ 1],
                                                         w.ctr + 16 * (par ^ 1)); count_launch(); }
            }
            PFF_CUDA(cudaMemsetAsync(w.ctr + 40, 0, 6 * sizeof(int), st));
            PFF_CUDA(cudaMemsetAsync(w.ctr + 50 + par, 0, sizeof(int), st));
            // it > 0 here means every earlier iteration took this path: labels only merged since
            const int *aprev = it == 0 ? nullptr : w.alist[par ^ 1];
            PFF_MODE_DISPATCH(bound_mode, l_saddle_lists, bid, is_border, z_prime, sad, basin_saddlenode, out, w.inv, z,
                              g, w.pits[par], np, w.blist, w.ctr + 40, aprev, w.ctr + 50 + (par ^ 1), w.alist[par],
                              w.ctr + 50 + par, grid, st);
        }
        if (!carve) {
            { k_carve_link_outlets<<<nbk, B, 0, st>>>(rec_, basin_saddlenode, out, N, 1); count_launch(); }  // :529
            PFF_TRY(check_cuda("pff_reroute_flow"));
            continue;
        }
        // ---- reroute_carve (:405-438) ----
        PFF_CUDA(cudaMemsetAsync(tag, 0, (size_t)N, st));
        PFF_CUDA(cudaMemsetAsync(tag_, 0, (size_t)N, st));
        if (general) {
            // the reference's tag propagation by pointer jumping (:424-435)
            { k_carve_tag_saddles<<<nbk, B, 0, st>>>(basin_saddlenode, tag, N); count_launch(); }
            PFF_CUDA(cudaMemcpyAsync(tag_, tag, (size_t)N, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemcpyAsync(rec, rec_, nb4, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemcpyAsync(rec__, rec_, nb4, cudaMemcpyDeviceToDevice, st));
            int *cflags = w.ctr + 192;
            PFF_CUDA(cudaMemsetAsync(cflags, 0, sizeof(int) * 64, st));
            const int carve_rounds = ceil_log2(N) + 2;
            for (int r = 0; r < carve_rounds; ++r) {
                { k_carve_it1<<<nbk, B, 0, st>>>(tag, tag_, rec, rec_, N, r, cflags); count_launch(); }
                { k_carve_it2<<<nbk, B, 0, st>>>(tag, tag_, rec, rec_, N, r, cflags); count_launch(); }
            }
            // finalise (:390-403): copy, reversal with the serial last writer, saddle links
            PFF_CUDA(cudaMemcpyAsync(rec, rec__, nb4, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemsetAsync(w.R, 0xff, nb4, st));  // claims start at -1
            { k_rev_claim<<<nbk, B, 0, st>>>(rec__, tag, w.R, N); count_launch(); }
            { k_rev_apply<<<nbk, B, 0, st>>>(rec, w.R, N); count_launch(); }
            { k_carve_link_outlets<<<nbk, B, 0, st>>>(rec, basin_saddlenode, out, N, 0); count_launch(); }
            PFF_CUDA(cudaMemcpyAsync(rec_, rec, nb4, cudaMemcpyDeviceToDevice, st));  // :526
            PFF_TRY(check_cuda("pff_reroute_flow"));
            continue;
        }
        // rec == rec_ here; rec__ holds the tile terminals of rec_
        { k_carve_segments<<<nsm * 4, 32 * SEG_WARPS, 0, st>>>(basin_saddlenode, rec_, rec__, w.pits[par], np, N,
                                                                 w.segs, w.ctr + 41, N, w.ctr + 43); count_launch(); }
        { k_carve_walk<<<nsm * 4, WALK_THREADS, 0, st>>>(rec_, rec, tag, tag_, w.segs, w.ctr + 41, N, nx, g.ny,
                                                          w.dirty); count_launch(); }
        { k_carve_link_list<<<grid, B, 0, st>>>(rec, basin_saddlenode, out, w.pits[par], np, N, w.dirty, nx); count_launch(); }
        // ---- next iteration: pits left, labels by basin relabelling, dirty tiles ----
        int *np_next = w.ctr + 16 * (par ^ 1);
        PFF_CUDA(cudaMemsetAsync(np_next, 0, 4 * sizeof(int), st));
        { k_relabel_init<<<grid, B, 0, st>>>(w.fin, bid, basin_saddlenode, out, w.pits[par], np, N, w.pits[par ^ 1],
                                             np_next, w.ctr + 45); count_launch(); }
        { k_dirty_list<<<div_up(ntiles, B), B, 0, st>>>(w.dirty, ntiles, w.tiles, w.ctr + 44); count_launch(); }
        // The basin relabelling, launched before the host reads this iteration's
        // flags so that one synchronisation serves both; its result is used only
        // if the loop goes on.  A basin chain that does not converge is a cycle.
        int *flags = w.ctr + 256;
        PFF_CUDA(cudaMemsetAsync(flags, 0, 64 * sizeof(int), st));
        static int coop_relabel = 0;
        if (!coop_relabel) {
            int per = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_relabel_jump_coop, 256, 0);
            coop_relabel = nsm * (per < 4 ? per : 4);
        }
        int *plist = w.pits[par];
        launch_relabel_jump_block(w.fin, plist, np, cudaGraphConditionalHandle{}, 0, st);
        void *args[] = {&w.fin, &plist, &np, &flags};
        PFF_CUDA(cudaLaunchCooperativeKernel((void *)k_relabel_jump_coop, coop_relabel, 256, args, 0, st));
        count_launch();
        int *cyc = w.ctr + 49;
        PFF_CUDA(cudaMemsetAsync(cyc, 0, sizeof(int), st));
        { k_relabel_check<<<grid, B, 0, st>>>(w.fin, out, w.pits[par], np, N, cyc); count_launch(); }
        int hv[5];
        PFF_TRY(read_ints(IntReads().add(w.ctr + 43, 3).add(np_next, 1).add(cyc, 1), hv, st));
        const int h[3] = {hv[0], hv[1], hv[2]}, hc = hv[4];
        nd_next = hv[3];
        // rec_ = rec on the carved cells (:526): inside the relabelling pass when
        // the loop goes on, else here
        if (h[0] || h[2] || it + 1 >= outer || hc || nd_next == 0) {
            { k_sync_tagged<<<div_up(div_up(N, 4), B), B, 0, st>>>(rec_, rec, tag, N, ((uintptr_t)tag & 3) == 0, nullptr); count_launch(); }
        }
        if (h[0]) break;  // walk bounds exceeded: reported below
        const int ndirty = h[1];
        if (h[2]) {
            // a reversed path without an outlet link (elevations >= 1e9 only)
            general = true;
            continue;
        }
        if (it + 1 >= outer) break;  // :500
        if (trace) fprintf(stderr, "[pff reroute]   after carve: next pits %d dirty %d cycle %d\n", nd_next, ndirty, hc);
        if (hc) {
            general = true;  // the carve closed a receiver cycle: the reference's path from here on
            continue;
        }
        if (nd_next == 0) {
            ++n_outer;  // the next iteration would count 0 pits, label, then break (:512-514)
            break;      // its labels are reset by basin_id_init (:537) anyway
        }
        { k_relabel<<<div_up(div_up(N, 4), B), B, 0, st>>>(bid, w.fin, rec_, rec, tag, tag_, N,
                                                           ((uintptr_t)bid & 15) == 0 && ((uintptr_t)tag & 3) == 0); count_launch(); }
        if (ndirty > 0)
            PFF_MODE_DISPATCH(g.mode, l_tile_terminal_list, rec_, rec__, w.R, w.ctr + 16 * par, g, w.tiles, w.ctr + 44,
                              std::min(ndirty, nsm * 8), st);
        incremental = true;
        PFF_TRY(check_cuda("pff_reroute_flow"));
    }
    int err[5] = {0, 0, 0, 0, 0};
    PFF_TRY(launch_basin_init(bid, g, st));  // :537
    PFF_TRY(read_ints(IntReads().add(w.ctr + 43, 5), err, st));
    if (err[0]) {
        set_error("pff_reroute_flow: carve walk exceeded its bounds");
        return PFF_ERR_NOCONV;
    }
    if (err[4]) {
        set_error("pff_reroute_flow: a receiver cycle longer than %d cells, or one whose serial labelling does not "
                  "converge to a single label", CYC_MAX);
        return PFF_ERR_NOCONV;
    }
    if (n_outer_out) *n_outer_out = n_outer;
    return check_cuda("pff_reroute_flow");
}

}  // namespace pff

// What the host does after the device-driven loop stopped in `state` (iteration it,
// bound outer, n_outer iterations counted): nothing for a finished loop, the
// reference's steps on the host for the general cases, an error otherwise.
static int reroute_after_graph(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                               float *z_prime, uint8_t *is_border, long long *out, long long *sad,
                               int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, const Grid &g, RerouteWs &w,
                               int state, int it, int outer, int n_outer, int *n_outer_out, cudaStream_t st)
{
    if (state == RR_NOPITS) return check_cuda("pff_reroute_flow");  // :496-497, bid untouched
    if (state == RR_GENERAL)  // non-D4 receivers or a receiver cycle in the input: the reference's steps
        return reroute_host_loop(bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, basin_saddlenode, tag, tag_,
                                 1, g, w, 0, 0, true, 0, n_outer_out, st);
    if (state == RR_RESUME)  // the carve closed a receiver cycle: the reference's steps from here on
        return reroute_host_loop(bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, basin_saddlenode, tag, tag_,
                                 1, g, w, it + 1, outer, true, n_outer, n_outer_out, st);
    if (state == RR_WALKERR) {
        set_error("pff_reroute_flow: carve walk exceeded its bounds");
        return PFF_ERR_NOCONV;
    }
    if (state != RR_DONE) {
        set_error("pff_reroute_flow: outer loop ended in state %d", state);
        return PFF_ERR_NOCONV;
    }
    if (n_outer_out) *n_outer_out = n_outer;
    return check_cuda("pff_reroute_flow");
}

extern "C" int pff_reroute_flow(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                                float *z_prime, uint8_t *is_border, int64_t *outlet, int64_t *basin_saddle,
                                int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int carve, int nx, int ny,
                                int bound_mode, const uint8_t *codes, void *workspace, size_t workspace_bytes,
                                int *n_outer_out, void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!bid || !rec || !rec_ || !rec__ || !z || !z_prime || !is_border || !outlet || !basin_saddle ||
        !basin_saddlenode || !tag || !tag_) {
        set_error("pff_reroute_flow: null pointer");
        return PFF_ERR_ARG;
    }
    const int N = nx * ny;
    if (!workspace || workspace_bytes < pff_reroute_workspace_bytes(N)) {
        set_error("pff_reroute_flow: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    Grid g{nx, ny, bound_mode, codes};
    cudaStream_t st = S(stream);
    RerouteWs w = carve_ws(workspace, workspace_bytes, N);
    long long *sad = (long long *)basin_saddle, *out = (long long *)outlet;
    const size_t nb4 = sizeof(int32_t) * (size_t)N;
    if (n_outer_out) *n_outer_out = 0;
    if (carve) {
        int state = 0, it = 0, outer = 0, n_outer = 0;
        const int rc = reroute_graph(bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, basin_saddlenode, tag,
                                     tag_, g, w, workspace, workspace_bytes, &state, &it, &outer, &n_outer, st);
        if (rc == PFF_OK)
            return reroute_after_graph(bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, basin_saddlenode, tag,
                                       tag_, g, w, state, it, outer, n_outer, n_outer_out, st);
        if (rc != PFF_ERR_UNSUPPORTED) return rc;
        clear_error();  // graphs unavailable: the host-driven loop below
    }
    PFF_CUDA(cudaMemcpyAsync(rec_, rec, nb4, cudaMemcpyDeviceToDevice, st));  // :491
    PFF_CUDA(cudaMemsetAsync(w.ctr, 0, 512 * sizeof(int), st));
    const int ntx = div_up(nx, TILE_W), ntiles = ntx * div_up(ny, TILE_H);
    PFF_CUDA(cudaMemsetAsync(w.dirty, 0, (size_t)ntiles, st));
    return reroute_host_loop(bid, rec, rec_, rec__, z, z_prime, is_border, out, sad, basin_saddlenode, tag, tag_,
                             carve, g, w, 0, 0, !carve, 0, n_outer_out, st);
}

extern "C" int pff_reroute_use_graphs(int on)
{
    clear_error();
    const int prev = rr_graphs_on() ? 1 : 0;
    g_rr_graphs.store(on != 0 ? 1 : 0);
    return prev;
}

// ---- asynchronous reroute ----------------------------------------------------------
// pff_reroute_flow split at its one synchronisation: the graph launch, whose last node
// copies the final state words into ctl_out, and the host's continuation from a host
// copy of those words.

#define PFF_REROUTE_ARGS                                                                                        \
    int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z, float *z_prime, uint8_t *is_border, \
        int64_t *outlet, int64_t *basin_saddle, int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int nx,  \
        int ny, int bound_mode, const uint8_t *codes, void *workspace, size_t workspace_bytes

static int reroute_args_ok(const char *who, PFF_REROUTE_ARGS)
{
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!bid || !rec || !rec_ || !rec__ || !z || !z_prime || !is_border || !outlet || !basin_saddle ||
        !basin_saddlenode || !tag || !tag_) {
        set_error("%s: null pointer", who);
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_reroute_workspace_bytes(nx * ny)) {
        set_error("%s: workspace too small", who);
        return PFF_ERR_WORKSPACE;
    }
    return PFF_OK;
}

// kernel counts of the last asynchronous launch per device (for the launch tally)
static RRKernelCounts g_async_kc[64];

extern "C" int pff_reroute_flow_async(PFF_REROUTE_ARGS, int *ctl_out, void *stream)
{
    clear_error();
    PFF_TRY(reroute_args_ok("pff_reroute_flow_async", bid, rec, rec_, rec__, z, z_prime, is_border, outlet,
                            basin_saddle, basin_saddlenode, tag, tag_, nx, ny, bound_mode, codes, workspace,
                            workspace_bytes));
    if (!ctl_out) {
        set_error("pff_reroute_flow_async: null ctl_out");
        return PFF_ERR_ARG;
    }
    Grid g{nx, ny, bound_mode, codes};
    RerouteWs w = carve_ws(workspace, workspace_bytes, nx * ny);
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    int state = 0, it = 0, outer = 0, n_outer = 0;
    RRKernelCounts kc{};
    const int rc = reroute_graph(bid, rec, rec_, rec__, z, z_prime, is_border, (long long *)outlet,
                                 (long long *)basin_saddle, basin_saddlenode, tag, tag_, g, w, workspace,
                                 workspace_bytes, &state, &it, &outer, &n_outer, S(stream), ctl_out, true, &kc);
    if (rc == PFF_ERR_UNSUPPORTED) {
        set_error("pff_reroute_flow_async: the device-driven loop is not available (graphs switched off or "
                  "not supported here); use pff_reroute_flow");
        return PFF_ERR_UNAVAILABLE;
    }
    PFF_TRY(rc);
    if (dev >= 0 && dev < 64) g_async_kc[dev] = kc;
    return PFF_OK;
}

extern "C" int pff_reroute_flow_finish(PFF_REROUTE_ARGS, const int *ctl_host, int *n_outer_out, void *stream)
{
    clear_error();
    PFF_TRY(reroute_args_ok("pff_reroute_flow_finish", bid, rec, rec_, rec__, z, z_prime, is_border, outlet,
                            basin_saddle, basin_saddlenode, tag, tag_, nx, ny, bound_mode, codes, workspace,
                            workspace_bytes));
    if (!ctl_host) {
        set_error("pff_reroute_flow_finish: null ctl_host");
        return PFF_ERR_ARG;
    }
    if (n_outer_out) *n_outer_out = 0;
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64) g_launches.fetch_add(rr_tally(g_async_kc[dev], ctl_host));
    Grid g{nx, ny, bound_mode, codes};
    RerouteWs w = carve_ws(workspace, workspace_bytes, nx * ny);
    return reroute_after_graph(bid, rec, rec_, rec__, z, z_prime, is_border, (long long *)outlet,
                               (long long *)basin_saddle, basin_saddlenode, tag, tag_, g, w, ctl_host[3], ctl_host[0],
                               ctl_host[1], ctl_host[2], n_outer_out, S(stream));
}

// ---- a region that runs only after a finished reroute ------------------------------------
// A graph: k_guard_set, then an IF node whose body is whatever the caller issues on
// its stream between pff_guard_begin and pff_guard_end.  The body runs when the
// reroute state in ctl[3] is "finished" (no pits, or done on the device) and the
// caller's flag (if any) is zero.

__global__ void k_guard_set(const int *ctl, const int *flag, cudaGraphConditionalHandle h)
{
    if (threadIdx.x) return;
    const int st = ctl[3];
    const bool go = (st == RR_NOPITS || st == RR_DONE) && (!flag || *flag == 0);
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

namespace {
struct Guard {
    cudaGraph_t G = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t capturing = nullptr;
    bool used = false;
};
constexpr int GUARDS = 1024;
std::mutex g_guard_mu;
Guard g_guards[GUARDS];
}  // namespace

extern "C" int pff_guard_begin(const int *ctl, const int *flag, void *stream, int *id)
{
    clear_error();
    if (!ctl || !id || !stream) {
        set_error("pff_guard_begin: bad arguments (a non-default stream is required)");
        return PFF_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_guard_mu);
    int k = 0;
    while (k < GUARDS && g_guards[k].used) ++k;
    if (k == GUARDS) {
        set_error("pff_guard_begin: too many guarded regions");
        return PFF_ERR_ARG;
    }
    Guard &gd = g_guards[k];
    PFF_CUDA(cudaGraphCreate(&gd.G, 0));
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, gd.G, 0, cudaGraphCondAssignDefault) != cudaSuccess) {
        cudaGraphDestroy(gd.G);
        gd.G = nullptr;
        return check_cuda("pff_guard_begin: conditional handle");
    }
    cudaKernelNodeParams kp{};
    void *args[] = {(void *)&ctl, (void *)&flag, (void *)&h};
    kp.func = (void *)k_guard_set;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
    kp.kernelParams = args;
    cudaGraphNode_t kn, cn;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    if (cudaGraphAddKernelNode(&kn, gd.G, nullptr, 0, &kp) != cudaSuccess ||
        cudaGraphAddNode(&cn, gd.G, &kn, 1, &cp) != cudaSuccess ||
        cudaStreamBeginCaptureToGraph(S(stream), cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed) != cudaSuccess) {
        cudaGraphDestroy(gd.G);
        gd.G = nullptr;
        return check_cuda("pff_guard_begin");
    }
    gd.capturing = S(stream);
    gd.used = true;
    *id = k;
    return PFF_OK;
}

extern "C" int pff_guard_end(int id, void *stream)
{
    clear_error();
    std::lock_guard<std::mutex> lk(g_guard_mu);
    if (id < 0 || id >= GUARDS || !g_guards[id].used || !g_guards[id].G || g_guards[id].capturing != S(stream)) {
        set_error("pff_guard_end: no region %d open on this stream", id);
        return PFF_ERR_ARG;
    }
    Guard &gd = g_guards[id];
    cudaGraph_t body = nullptr;
    const cudaError_t e = cudaStreamEndCapture(gd.capturing, &body);
    gd.capturing = nullptr;
    if (e == cudaSuccess && cudaGraphInstantiate(&gd.exec, gd.G, 0) == cudaSuccess) return PFF_OK;
    set_error("pff_guard_end: %s", cudaGetErrorString(e != cudaSuccess ? e : cudaGetLastError()));
    cudaGetLastError();
    cudaGraphDestroy(gd.G);
    gd = Guard{};
    return PFF_ERR_CUDA;
}

extern "C" int pff_guard_launch(int id, void *stream)
{
    clear_error();
    cudaGraphExec_t exec = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_guard_mu);
        if (id >= 0 && id < GUARDS && g_guards[id].used) exec = g_guards[id].exec;
    }
    if (!exec) {
        set_error("pff_guard_launch: region %d is not complete", id);
        return PFF_ERR_ARG;
    }
    PFF_CUDA(cudaGraphLaunch(exec, S(stream)));
    return PFF_OK;
}

extern "C" int pff_guard_destroy(int id)
{
    clear_error();
    std::lock_guard<std::mutex> lk(g_guard_mu);
    if (id < 0 || id >= GUARDS || !g_guards[id].used) {
        set_error("pff_guard_destroy: no region %d", id);
        return PFF_ERR_ARG;
    }
    Guard &gd = g_guards[id];
    if (gd.capturing) {
        cudaGraph_t body = nullptr;
        cudaStreamEndCapture(gd.capturing, &body);
    }
    if (gd.exec) cudaGraphExecDestroy(gd.exec);
    if (gd.G) cudaGraphDestroy(gd.G);
    gd = Guard{};
    cudaGetLastError();
    return PFF_OK;
}

// flag[0] = 1 if (double)val[0] / div < thr, else 0: the host's residual test
// (float(value) / dt < threshold, in double) made on the device
__global__ void k_residual_flag(const float *val, double div, double thr, int *flag)
{
    if (threadIdx.x == 0) flag[0] = ((double)val[0] / div < thr) ? 1 : 0;
}

// out_dev[0] (if given) and out_host[0] (pinned host memory, written through its
// unified address; if given) = val[0]: one kernel instead of two copies
__global__ void k_value_store(const float *val, float *out_dev, float *out_host)
{
    if (threadIdx.x) return;
    const float v = val[0];
    if (out_dev) out_dev[0] = v;
    if (out_host) *(volatile float *)out_host = v;
}

extern "C" int pff_value_store(const float *val, float *out_dev, float *out_host, void *stream)
{
    clear_error();
    if (!val) {
        set_error("pff_value_store: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_value_store<<<1, 32, 0, S(stream)>>>(val, out_dev, out_host); count_launch(); }
    return check_cuda("pff_value_store");
}

extern "C" int pff_residual_flag(const float *val, double div, double thr, int *flag, void *stream)
{
    clear_error();
    if (!val || !flag) {
        set_error("pff_residual_flag: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_residual_flag<<<1, 32, 0, S(stream)>>>(val, div, thr, flag); count_launch(); }
    return check_cuda("pff_residual_flag");
}
