// libpff drainage accumulation by hierarchical tile contraction: the upstream sums
// that pyfastflow's accumulate_constant_Q forms by rake and compress
// (pyfastflow/flow/downstream_propag.py:21-179 driven by flow/flowfields.py:254-292),
// computed with a different decomposition.
//
// Q[i] = sum of the seeds of every cell whose receiver path passes through i
// (i included); counts[i] = the number of such cells.  The sums are formed
// exactly: counts as uint32, seeds as 64-bit fixed point (seed * 2^s rounded to
// an integer, with s chosen from max|seed| so that no sum can overflow), and Q is
// the fixed-point total rounded once to f32.  Integer sums do not depend on the
// order of additions, so the result is deterministic although every level uses
// atomics.  The reference's f32 rake-and-compress sums differ from the exact sum
// by their own rounding: counts are identical, Q agrees to f32 rounding.
//
// Decomposition (each level is one kernel launch up and one down):
//   level 0   32 x 32 cell tiles, one CTA each.  In shared memory every cell's
//             in-tile upstream sum is formed by pointer doubling (below): about
//             log2 of the longest in-tile path rounds, every cell busy in every
//             round, no serial chain.  Cells whose receiver lies in another tile
//             ("exits") become the nodes of level 1, carrying their in-tile totals.
//   level L   blocks of S_L x S_L tiles (S_1 = 8, S_{L+1} = 2 S_L).  A node's
//             parent at level L is the terminal (within the lower-level block) of
//             the cell or node its flow enters; pointer-doubling rounds run over
//             a block's nodes in shared memory.  Nodes whose parent lies in another block are
//             the next level's nodes.  The top level is one block over the grid.
//   down      from the top: each level's nodes receive the totals of the nodes of
//             the level above that drain into them (integer atomics), and the walks
//             run again with those inflows added to the seeds, giving every node
//             its full total; level 0 then gives every cell its full total.
// A receiver cycle shows as a successor pointer that outlives the rounds; it is
// reported in the status word (the result is then unspecified).
#include <algorithm>
#include <cmath>
#include "pff_internal.h"

namespace pff {

constexpr int TR_T = 32;                 // tile side in cells
constexpr int TR_TC = TR_T * TR_T;       // cells per tile
constexpr int TR_T0_THREADS = 256;
constexpr int TR_LB_THREADS = 1024;
constexpr int TR_S1 = 8;                 // level-1 block side in tiles
constexpr int TR_MAXLEV = 20;
constexpr int TR_SMEM_NODES = 8192;      // nodes of a block kept in shared memory
constexpr int TR_NODE_BYTES = 24;        // lo, hi, cnt, lpar, jmp, tn

// status bits
constexpr int TR_ERR_RCV = 1;       // a receiver index out of range
constexpr int TR_ERR_CYCLE = 2;     // a receiver cycle
constexpr int TR_ERR_CAP = 4;       // more exits in a tile than the capacity (local = 0 only)
constexpr int TR_ERR_NONLOCAL = 8;  // local = 1 but a receiver leads into another tile's interior
constexpr int TR_ERR_SEED = 16;     // a non-finite seed

struct TreeLevel {
    long long *W;        // in-block total carried up (fixed point)
    unsigned *C;         // in-block count carried up
    int *rawpar;         // parent before resolution (level 1: a cell; else a position one level down)
    int *par;            // resolved parent position at this level, or -1
    int *up;             // position at the next level of this node's block terminal, or -1
    long long *In;       // inflow from the level above (fixed point)
    unsigned *Inc;       // inflow count
    int *src;            // position of this node one level down (levels >= 2)
    int *cnt;            // nodes per block (appended by the level below)
    int side;            // block side in tiles
    int nbx, nby;        // blocks per row / column
};

struct TreeArgs {
    int nx, ny, ntx, nty, N;
    int slots;           // node slots per level (tiles x cap0)
    int cap0;            // node slots per tile
    int nlev;            // block levels 1..nlev (nlev = top)
    int local;           // receivers lead only to tile-perimeter cells of other tiles
    unsigned char *marker;  // cell receives inflow from another tile this call
    long long *In0;
    unsigned *Inc0;
    int *up0;            // per cell: level-1 position of its tile terminal, or -1
    int *status;         // [0] error bits, [1] max |seed| bits
    long long *scr_acc;  // fallback storage for blocks larger than TR_SMEM_NODES
    unsigned *scr_cnt;
    int *scr_lpar, *scr_pend, *scr_tn;
    long long *scr_acc2;  // start-of-round copies for those blocks
    unsigned *scr_cnt2;
    TreeLevel lv[TR_MAXLEV + 1];
};

// ---- block geometry (row-major blocks, closed-form tile offsets) ------------------
struct BlockGeo {
    int tile_off;   // first tile index of the block in the level's slot order
    int tiles;      // tiles in the block
};
__host__ __device__ __forceinline__ BlockGeo block_geo(int bx, int by, int side, int ntx, int nty)
{
    const int h = min(side, nty - by * side), w = min(side, ntx - bx * side);
    BlockGeo g;
    g.tile_off = by * side * ntx + bx * side * h;
    g.tiles = w * h;
    return g;
}

// ---- fixed point --------------------------------------------------------------------
// s such that N * max|seed| * 2^s < 2^62: no partial sum can overflow int64.
__device__ __forceinline__ int fixed_shift(unsigned maxbits, int N)
{
    const float m = __uint_as_float(maxbits);
    if (!(m > 0.f)) return 0;
    int e;
    const unsigned E = (maxbits >> 23) & 0xffu;
    if (E) e = (int)E - 126;    // m = f * 2^e with f in [0.5, 1): m < 2^e
    else frexpf(m, &e);
    const int nb = 32 - __clz(N);  // N < 2^nb
    return 62 - (e + nb);
}
// round(w * 2^s) to the nearest integer, ties to even, from the IEEE-754 fields:
// w = +-m * 2^(E-150) (m with its implicit bit; E = 0: m * 2^-149).  Exact in
// 64 bits for every |w| <= max|seed| (fixed_shift keeps m * 2^(e+s) < 2^62).
__device__ __forceinline__ long long to_fixed(float w, int s)
{
    const unsigned b = __float_as_uint(w);
    const unsigned E = (b >> 23) & 0xffu;
    unsigned long long m = b & 0x7fffffu;
    int e;
    if (E) { m |= 0x800000u; e = (int)E - 150; }
    else e = -149;
    const int sh = e + s;
    unsigned long long v;
    if (sh >= 0) v = sh < 40 ? m << sh : 0;  // (larger shifts only for non-finite seeds, flagged elsewhere)
    else {
        const int k = -sh;
        if (k > 40) v = 0;
        else {
            const unsigned long long q = m >> k, rem = m & ((1ull << k) - 1), half = 1ull << (k - 1);
            v = q + ((rem > half || (rem == half && (q & 1))) ? 1 : 0);
        }
    }
    return (b >> 31) ? -(long long)v : (long long)v;
}
__device__ __forceinline__ float from_fixed(long long v, int s)
{
    // one correct rounding to f32, then an exact power-of-two scaling
    float f = __ll2float_rn(v);
    while (s > 126) { f = __fmul_rn(f, 0x1p-126f); s -= 126; }
    while (s < -126) { f = __fmul_rn(f, 0x1p126f); s += 126; }
    return __fmul_rn(f, __int_as_float((127 - s) << 23));
}

// max |seed| over the grid (as f32 bits: non-negative floats order as integers)
__global__ void k_tree_seedmax(const float *__restrict__ w, int N, int *status)
{
    unsigned m = 0;
    bool bad = false;
    auto take = [&](float x) {
        const float a = fabsf(x);
        if (!(a <= 3.4028235e38f)) bad = true;
        else m = max(m, __float_as_uint(a));
    };
    const int stride = gridDim.x * blockDim.x, t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (((uintptr_t)w & 15) == 0) {  // 16-byte loads, then the tail
        const float4 *w4 = reinterpret_cast<const float4 *>(w);
        for (int q = t0; q < N / 4; q += stride) {
            const float4 v = __ldg(w4 + q);
            take(v.x); take(v.y); take(v.z); take(v.w);
        }
        for (int i = (N / 4) * 4 + t0; i < N; i += stride) take(w[i]);
    } else {
        for (int i = t0; i < N; i += stride) take(w[i]);
    }
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax((unsigned *)&status[1], m);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&status[0], TR_ERR_SEED);
}

// ---- accumulation by pointer doubling -------------------------------------------------------
// Within a block, with A the donor -> receiver adjacency restricted to the block,
// the upstream sums are Q = sum_j A^j w = prod_i (I + A^(2^i)) w (A is nilpotent
// on a forest).  Round i applies (I + A^(2^i)): every node adds its current sum
// to the node 2^i steps downstream (integer atomics), and the successor pointers
// double; a pointer dies when its path leaves the block or ends at a root.  All
// nodes work in every round, so there is no serial chain; the rounds stop when
// every pointer is dead (after ceil(log2 of the longest in-block path) rounds).
// A pointer still alive after log2(n) + 1 rounds lies on a receiver cycle.
//
// jmp[k]: successor 2^i steps down, or -1.  Register copies of each thread's
// nodes (RPT per thread) hold the start-of-round values.
template <int RPT, int NT>
__device__ __forceinline__ bool doubling_rounds(int n, int *jmp, unsigned *lo, unsigned *hi, unsigned *cnt,
                                                int max_rounds)
{
    // totals as 32-bit halves: the low half's atomic returns the old value, and the
    // adder that wraps it carries into the high half (each wrap counted once)
    for (int r = 0; r < max_rounds; ++r) {
        int sj[RPT], nj[RPT];
        unsigned sl[RPT], sh[RPT], sc[RPT];
        bool live = false;
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int k = threadIdx.x + j * NT;
            sj[j] = -1;
            if (k < n) {
                sj[j] = jmp[k];
                if (sj[j] >= 0) {
                    sl[j] = lo[k];
                    sh[j] = hi[k];
                    sc[j] = cnt[k];
                    nj[j] = jmp[sj[j]];
                    live = true;
                }
            }
        }
        if (!__syncthreads_or(live)) return true;
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            if (sj[j] >= 0) {
                const int k = threadIdx.x + j * NT;
                const unsigned old = atomicAdd(&lo[sj[j]], sl[j]);
                atomicAdd(&hi[sj[j]], sh[j] + (old + sl[j] < old ? 1u : 0u));
                atomicAdd(&cnt[sj[j]], sc[j]);
                jmp[k] = nj[j];
            }
        }
        __syncthreads();
    }
    // a pointer that is still alive: a path longer than the block (a cycle)
    bool live = false;
    for (int k = threadIdx.x; k < n; k += NT) live |= jmp[k] >= 0;
    return !__syncthreads_or(live);
}

// ---- level 0: one CTA per tile ---------------------------------------------------------------
// The same doubling rounds as doubling_rounds(), with each 64-bit total held as
// two 32-bit halves in shared memory: 32-bit shared atomics are single
// operations, 64-bit ones are not.  The low half's atomic returns the old value,
// so the adder whose addition wraps it adds the carry to the high half; every
// wrap is counted exactly once, and the 64-bit sum is exact.
//
// DOWN = false: in-tile totals, level-1 nodes for the exits, up0 for the cells
// other tiles can drain into.  DOWN = true: totals with the inflows, written as
// Q (f32) and counts.
template <bool DOWN>
__global__ void __launch_bounds__(TR_T0_THREADS) k_tree_tile(const int32_t *__restrict__ rcv,
                                                             const float *__restrict__ w, float value,
                                                             float *Q, unsigned *counts, TreeArgs a)
{
    constexpr int RPT = TR_TC / TR_T0_THREADS;
    __shared__ unsigned lo[TR_TC], hi[TR_TC];
    __shared__ unsigned cnt[TR_TC];
    __shared__ int jmp[TR_TC];
    __shared__ int lpar[TR_TC];  // -2 no cell, -1 root, -3 exit, else in-tile receiver
    __shared__ int s_n, s_base, s_err;
    const int tile = blockIdx.x;
    const int tx = tile % a.ntx, ty = tile / a.ntx;
    const int x0 = tx * TR_T, y0 = ty * TR_T;
    const int tw = min(TR_T, a.nx - x0), th = min(TR_T, a.ny - y0);
    const int s = fixed_shift(w ? (unsigned)a.status[1] : __float_as_uint(fabsf(value)), a.N);
    const long long cval = w ? 0 : to_fixed(value, s);
    if (threadIdx.x == 0) { s_n = 0; s_err = 0; }
    for (int k = threadIdx.x; k < TR_TC; k += TR_T0_THREADS) {
        const int lx = k & (TR_T - 1), ly = k >> 5;
        int lp = -2;
        unsigned long long sv = 0;
        unsigned sc = 0;
        if (lx < tw && ly < th) {
            const int gi = (y0 + ly) * a.nx + x0 + lx;
            int r = rcv[gi];
            if (r < 0 || r >= a.N) { atomicOr(&s_err, TR_ERR_RCV); r = gi; }
            const int d = r - gi;
            if (d == 0) lp = -1;
            else if (d == 1 && lx + 1 < tw) lp = k + 1;  // D4 neighbours without a division
            else if (d == -1 && lx > 0) lp = k - 1;
            else if (d == a.nx && ly + 1 < th) lp = k + TR_T;
            else if (d == -a.nx && ly > 0) lp = k - TR_T;
            else {
                const int ry = r / a.nx, rx = r - ry * a.nx;
                lp = (rx >= x0 && rx < x0 + tw && ry >= y0 && ry < y0 + th) ? (ry - y0) * TR_T + rx - x0 : -3;
            }
            sv = (unsigned long long)(w ? to_fixed(w[gi], s) : cval);
            sc = 1;
            if (DOWN && a.marker[gi]) {
                sv += (unsigned long long)a.In0[gi];
                sc += a.Inc0[gi];
            }
        }
        lpar[k] = lp;
        jmp[k] = lp >= 0 ? lp : -1;
        lo[k] = (unsigned)sv;
        hi[k] = (unsigned)(sv >> 32);
        cnt[k] = sc;
    }
    __syncthreads();
    // doubling rounds: the longest in-tile path is < 1024 = 2^10 cells
    bool cyc = false;
    unsigned alive = 0;  // this thread's cells whose pointer is still alive
#pragma unroll
    for (int j = 0; j < RPT; ++j) alive |= (jmp[threadIdx.x + j * TR_T0_THREADS] >= 0 ? 1u : 0u) << j;
    for (int r = 0;; ++r) {
        int sj[RPT], nj[RPT];
        unsigned sl[RPT], sh[RPT], sc[RPT];
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            const int k = threadIdx.x + j * TR_T0_THREADS;
            sj[j] = -1;
            if (alive >> j & 1u) {
                sj[j] = jmp[k];
                sl[j] = lo[k];
                sh[j] = hi[k];
                sc[j] = cnt[k];
                nj[j] = jmp[sj[j]];
                if (nj[j] < 0) alive &= ~(1u << j);
            }
        }
        if (!__syncthreads_or(sj[0] >= 0 || sj[1] >= 0 || sj[2] >= 0 || sj[3] >= 0)) break;
        if (r == 10) { cyc = true; break; }  // a path longer than the tile: a cycle
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            if (sj[j] >= 0) {
                const int k = threadIdx.x + j * TR_T0_THREADS;
                const unsigned old = atomicAdd(&lo[sj[j]], sl[j]);
                atomicAdd(&hi[sj[j]], sh[j] + (old + sl[j] < old ? 1u : 0u));
                atomicAdd(&cnt[sj[j]], sc[j]);
                jmp[k] = nj[j];
            }
        }
        __syncthreads();
    }
    if (cyc && threadIdx.x == 0) s_err |= TR_ERR_CYCLE;

    if (DOWN) {
        for (int k = threadIdx.x; k < TR_TC; k += TR_T0_THREADS) {
            const int lx = k & (TR_T - 1), ly = k >> 5;
            if (lx < tw && ly < th) {
                const int gi = (y0 + ly) * a.nx + x0 + lx;
                if (Q) Q[gi] = from_fixed((long long)(((unsigned long long)hi[k] << 32) | lo[k]), s);
                if (counts) counts[gi] = cnt[k];
                a.marker[gi] = 0;  // leave the markers clear for the next call
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_err) atomicOr(&a.status[0], s_err);
        return;
    }

    // exits -> level-1 nodes of this tile's level-1 block
    const TreeLevel &L1 = a.lv[1];
    const int bx = tx / L1.side, by = ty / L1.side;
    const int b1 = by * L1.nbx + bx;
    const BlockGeo g1 = block_geo(bx, by, L1.side, a.ntx, a.nty);
    int mine = 0;
    for (int k = threadIdx.x; k < TR_TC; k += TR_T0_THREADS) mine += lpar[k] == -3;
    for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&s_n, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        s_base = s_n ? atomicAdd(&L1.cnt[b1], s_n) : 0;
        if (s_base + s_n > g1.tiles * a.cap0) { s_err |= TR_ERR_CAP; s_n = -1; }
        s_n = s_n < 0 ? -1 : 0;  // reused as the rank counter below (-1: no room)
    }
    __syncthreads();
    const int slot0 = g1.tile_off * a.cap0 + s_base;
    int *q = jmp;  // free after the rounds: level-1 position of each exit
    for (int k = threadIdx.x; k < TR_TC; k += TR_T0_THREADS) {
        int qk = -1;
        if (lpar[k] == -3 && s_n >= 0) {
            const int lx = k & (TR_T - 1), ly = k >> 5;
            const int gi = (y0 + ly) * a.nx + x0 + lx;
            const int r = rcv[gi];
            qk = slot0 + atomicAdd(&s_n, 1);
            L1.W[qk] = (long long)(((unsigned long long)hi[k] << 32) | lo[k]);
            L1.C[qk] = cnt[k];
            L1.rawpar[qk] = r;
            L1.src[qk] = gi;
            a.In0[r] = 0;
            a.Inc0[r] = 0;
            a.marker[r] = 1;
            if (a.local) {  // the entry must be on the perimeter of its own tile
                const int ry = r / a.nx, rx = r - ry * a.nx;
                const int ex = rx % TR_T, ey = ry % TR_T;
                if (!(ex == 0 || ey == 0 || ex == TR_T - 1 || ey == TR_T - 1 || rx == a.nx - 1 || ry == a.ny - 1))
                    atomicOr(&s_err, TR_ERR_NONLOCAL);
            }
        }
        q[k] = qk;
    }
    __syncthreads();
    // up0 = level-1 position of the cell's tile terminal (if that is an exit), for
    // the cells another tile's exit can enter: the perimeter when local, every cell
    // otherwise; each walks down to its terminal
    const int per = a.local ? (tw + tw + max(th - 2, 0) * 2 - (th == 1 ? tw : 0)) : tw * th;
    for (int e = threadIdx.x; e < per; e += TR_T0_THREADS) {
        int lx, ly;
        if (!a.local) { ly = e / tw; lx = e - ly * tw; }
        else if (e < tw) { lx = e; ly = 0; }
        else if (e < 2 * tw && th > 1) { lx = e - tw; ly = th - 1; }
        else { const int f = e - 2 * tw; lx = (f & 1) ? tw - 1 : 0; ly = 1 + (f >> 1); }
        int t = ly * TR_T + lx;
        for (int st = 0; st < TR_TC && lpar[t] >= 0; ++st) t = lpar[t];
        a.up0[(y0 + ly) * a.nx + x0 + lx] = lpar[t] == -3 ? q[t] : -1;
    }
    if (threadIdx.x == 0 && s_err) atomicOr(&a.status[0], s_err);
}

// ---- levels >= 1: one CTA per block -----------------------------------------------------------
// MODE 0 up (local totals, next-level nodes, up pointers), 1 down (totals with the
// inflows, scattered one level down), 2 top (up with no exits, then scattered).
template <int MODE>
__global__ void __launch_bounds__(TR_LB_THREADS) k_tree_level(int L, TreeArgs a)
{
    extern __shared__ __align__(16) unsigned char tsm[];
    __shared__ int s_n, s_base, s_err;
    const TreeLevel &V = a.lv[L];
    const int b = blockIdx.x;
    const int bx = b % V.nbx, by = b / V.nbx;
    const BlockGeo g = block_geo(bx, by, V.side, a.ntx, a.nty);
    const int base = g.tile_off * a.cap0;
    const int n = min(V.cnt[b], g.tiles * a.cap0);  // appends past the capacity were refused and flagged
    if (n <= 0) return;
    unsigned *lo, *hi;  // totals as 32-bit halves
    unsigned *cnt;
    int *lpar, *jmp, *tn;
    const bool in_smem = n <= TR_SMEM_NODES;
    if (in_smem) {
        lo = (unsigned *)tsm;
        hi = lo + TR_SMEM_NODES;
        cnt = hi + TR_SMEM_NODES;
        lpar = (int *)(cnt + TR_SMEM_NODES);
        jmp = lpar + TR_SMEM_NODES;
        tn = jmp + TR_SMEM_NODES;
    } else {  // a block too large for shared memory works in its slice of the scratch
        lo = (unsigned *)a.scr_acc + base;  // scr_acc: 2 S unsigned
        hi = (unsigned *)a.scr_acc + a.slots + base;
        cnt = a.scr_cnt + base;
        lpar = a.scr_lpar + base;
        jmp = a.scr_pend + base;
        tn = a.scr_tn + base;
    }
    if (threadIdx.x == 0) { s_n = 0; s_err = 0; }
    for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
        const int pos = base + k;
        int p;
        if (MODE == 1) {
            p = V.par[pos];
        } else {
            const int rp = V.rawpar[pos];
            if (rp < 0 || rp >= (L == 1 ? a.N : a.slots)) {
                atomicOr(&s_err, TR_ERR_RCV);
                p = -1;
            } else {
                p = L == 1 ? a.up0[rp] : a.lv[L - 1].up[rp];
            }
            if (p < -1 || p >= a.slots) {  // an entry that was never given a terminal (local = 1 violated)
                atomicOr(&s_err, TR_ERR_NONLOCAL);
                p = -1;
            }
            V.par[pos] = p;
        }
        const int lp = p < 0 ? -1 : (p >= base && p < base + n ? p - base : -3);
        lpar[k] = lp;
        jmp[k] = lp >= 0 ? lp : -1;
        unsigned long long sv = (unsigned long long)V.W[pos];
        unsigned sc = V.C[pos];
        if (MODE == 1) {
            sv += (unsigned long long)V.In[pos];
            sc += V.Inc[pos];
        } else {
            V.In[pos] = 0;
            V.Inc[pos] = 0;
        }
        lo[k] = (unsigned)sv;
        hi[k] = (unsigned)(sv >> 32);
        cnt[k] = sc;
    }
    __syncthreads();
    int rounds = 1;
    while ((1 << rounds) < n) ++rounds;
    bool ok;
    if (in_smem) {
        ok = doubling_rounds<TR_SMEM_NODES / TR_LB_THREADS, TR_LB_THREADS>(n, jmp, lo, hi, cnt, rounds + 1);
    } else {
        // the same rounds with the start-of-round values in a second scratch (tn holds the next pointers)
        ok = true;
        for (int r = 0;; ++r) {
            bool live = false;
            for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
                const int j = jmp[k];
                tn[k] = j >= 0 ? jmp[j] : -1;
                live |= j >= 0;
            }
            if (!__syncthreads_or(live)) break;
            if (r > rounds) { ok = false; break; }
            for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {  // start-of-round snapshot
                const int j = jmp[k];
                if (j >= 0) {
                    a.scr_acc2[base + k] = (long long)(((unsigned long long)hi[k] << 32) | lo[k]);
                    a.scr_cnt2[base + k] = cnt[k];
                }
            }
            __syncthreads();
            for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
                const int j = jmp[k];
                if (j >= 0) {
                    const unsigned long long x = (unsigned long long)a.scr_acc2[base + k];
                    const unsigned old = atomicAdd(&lo[j], (unsigned)x);
                    atomicAdd(&hi[j], (unsigned)(x >> 32) + (old + (unsigned)x < old ? 1u : 0u));
                    atomicAdd(&cnt[j], a.scr_cnt2[base + k]);
                }
            }
            __syncthreads();
            for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) jmp[k] = tn[k];
            __syncthreads();
        }
    }
    if (!ok && threadIdx.x == 0) s_err |= TR_ERR_CYCLE;
    __syncthreads();

    if (MODE != 0) {
        // every node of this level drains into a node one level down (in another
        // block of that level): add its total to that node's inflow
        for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
            const int pos = base + k;
            if (L == 1) {
                const int cell = V.rawpar[pos];
                if (cell < 0 || cell >= a.N) continue;  // flagged in the up pass
                atomicAdd((unsigned long long *)&a.In0[cell], ((unsigned long long)hi[k] << 32) | lo[k]);
                atomicAdd(&a.Inc0[cell], cnt[k]);
            } else {
                const TreeLevel &D = a.lv[L - 1];
                const int sp = V.src[pos];
                const int t = (sp >= 0 && sp < a.slots) ? D.par[sp] : -1;
                if (t < 0 || t >= a.slots) continue;
                atomicAdd((unsigned long long *)&D.In[t], ((unsigned long long)hi[k] << 32) | lo[k]);
                atomicAdd(&D.Inc[t], cnt[k]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0 && s_err) atomicOr(&a.status[0], s_err);
        return;
    }

    // up: block terminals, then the exits become nodes of the next level
    for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) tn[k] = lpar[k] >= 0 ? lpar[k] : k;
    __syncthreads();
    for (int r = 0; r <= rounds; ++r) {
        bool ch = false;
        for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
            const int t = tn[k], tt = tn[t];
            if (tt != t) { tn[k] = tt; ch = true; }
        }
        if (!__syncthreads_or(ch)) break;
    }
    const TreeLevel &U = a.lv[L + 1];
    const int ubx = bx / 2, uby = by / 2;
    const int ub = uby * U.nbx + ubx;
    const BlockGeo ug = block_geo(ubx, uby, U.side, a.ntx, a.nty);
    int mine = 0;
    for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) mine += lpar[k] == -3;
    for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&s_n, mine);
    __syncthreads();
    if (threadIdx.x == 0) {
        s_base = s_n ? atomicAdd(&U.cnt[ub], s_n) : 0;
        if (s_base + s_n > ug.tiles * a.cap0) { s_err |= TR_ERR_CAP; s_n = -1; }
        s_n = s_n < 0 ? -1 : 0;
    }
    __syncthreads();
    const int slot0 = ug.tile_off * a.cap0 + s_base;
    for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
        int q = -1;
        if (lpar[k] == -3 && s_n >= 0) {
            const int pos = base + k;
            q = slot0 + atomicAdd(&s_n, 1);
            U.W[q] = (long long)(((unsigned long long)hi[k] << 32) | lo[k]);
            U.C[q] = cnt[k];
            U.rawpar[q] = V.par[pos];
            U.src[q] = pos;
        }
        jmp[k] = q;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += TR_LB_THREADS) {
        const int t = tn[k];
        V.up[base + k] = lpar[t] == -3 ? jmp[t] : -1;
    }
    if (threadIdx.x == 0 && s_err) atomicOr(&a.status[0], s_err);
}

// ---- host --------------------------------------------------------------------------------------
struct TreePlan {
    int ntx, nty, ntiles, nlev, cap0;
    long long slots;
    int nb[TR_MAXLEV + 1], nbx[TR_MAXLEV + 1], nby[TR_MAXLEV + 1], side[TR_MAXLEV + 1];
};

static TreePlan tree_plan(int nx, int ny, int local)
{
    TreePlan p{};
    p.ntx = (nx + TR_T - 1) / TR_T;
    p.nty = (ny + TR_T - 1) / TR_T;
    p.ntiles = p.ntx * p.nty;
    p.cap0 = local ? 128 : 256;
    p.slots = (long long)p.ntiles * p.cap0;
    int side = TR_S1, L = 1;
    for (;;) {
        p.side[L] = side;
        p.nbx[L] = (p.ntx + side - 1) / side;
        p.nby[L] = (p.nty + side - 1) / side;
        p.nb[L] = p.nbx[L] * p.nby[L];
        if (p.nb[L] == 1 || L == TR_MAXLEV - 1) break;
        side *= 2;
        ++L;
    }
    p.nlev = L;
    return p;
}

static size_t tree_bytes(const TreePlan &p, int N)
{
    const size_t S = (size_t)p.slots;
    size_t b = 0;
    b += Carver::round((size_t)N) + Carver::round(8 * (size_t)N) + 2 * Carver::round(4 * (size_t)N);  // level 0
    b += Carver::round(sizeof(int) * 64);                                                             // status
    b += 2 * Carver::round(8 * S) + 5 * Carver::round(4 * S);                                         // scratch
    for (int L = 1; L <= p.nlev; ++L)
        b += 2 * Carver::round(8 * S) + 6 * Carver::round(4 * S) + Carver::round(sizeof(int) * (size_t)p.nb[L]);
    return b + 4096;
}

}  // namespace pff

using namespace pff;

extern "C" size_t pff_accumulate_tree_workspace_bytes(int nx, int ny, int local)
{
    if (nx < 1 || ny < 1 || (long long)nx * ny > (1LL << 30)) return 0;
    return tree_bytes(tree_plan(nx, ny, local), nx * ny);
}

extern "C" int pff_accumulate_tree(const int32_t *receivers, const float *weights, float value, float *Q,
                                   uint32_t *counts, int nx, int ny, int local, void *workspace,
                                   size_t workspace_bytes, void *stream)
{
    clear_error();
    if (nx < 1 || ny < 1 || (long long)nx * ny > (1LL << 30) || !receivers || (!Q && !counts)) {
        set_error("pff_accumulate_tree: bad arguments");
        return PFF_ERR_ARG;
    }
    const int N = nx * ny;
    const TreePlan p = tree_plan(nx, ny, local);
    if (!workspace || workspace_bytes < tree_bytes(p, N)) {
        set_error("pff_accumulate_tree: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    if (!weights && !(fabsf(value) <= 3.4028235e38f)) {
        set_error("pff_accumulate_tree: non-finite seed value");
        return PFF_ERR_ARG;
    }
    cudaStream_t st = S(stream);
    Carver cv(workspace, workspace_bytes);
    TreeArgs a{};
    a.nx = nx; a.ny = ny; a.ntx = p.ntx; a.nty = p.nty; a.N = N;
    a.cap0 = p.cap0; a.nlev = p.nlev; a.local = local ? 1 : 0;
    a.slots = (int)p.slots;
    a.marker = cv.take<unsigned char>(N);
    a.In0 = cv.take<long long>(N);
    a.Inc0 = cv.take<unsigned>(N);
    a.up0 = cv.take<int>(N);
    a.status = cv.take<int>(64);
    const size_t S = (size_t)p.slots;
    a.scr_acc = cv.take<long long>(S);
    a.scr_cnt = cv.take<unsigned>(S);
    a.scr_lpar = cv.take<int>(S);
    a.scr_pend = cv.take<int>(S);
    a.scr_tn = cv.take<int>(S);
    a.scr_acc2 = cv.take<long long>(S);
    a.scr_cnt2 = cv.take<unsigned>(S);
    for (int L = 1; L <= p.nlev; ++L) {
        TreeLevel &V = a.lv[L];
        V.W = cv.take<long long>(S);
        V.In = cv.take<long long>(S);
        V.C = cv.take<unsigned>(S);
        V.Inc = cv.take<unsigned>(S);
        V.rawpar = cv.take<int>(S);
        V.par = cv.take<int>(S);
        V.up = cv.take<int>(S);
        V.src = cv.take<int>(S);
        V.cnt = cv.take<int>(p.nb[L]);
        V.side = p.side[L];
        V.nbx = p.nbx[L];
        V.nby = p.nby[L];
    }
    // the top level's exits would go to level nlev+1: there are none (one block)
    a.lv[p.nlev + 1] = a.lv[p.nlev];

    PFF_CUDA(cudaMemsetAsync(a.marker, 0, (size_t)N, st));
    PFF_CUDA(cudaMemsetAsync(a.status, 0, sizeof(int) * 64, st));
    for (int L = 1; L <= p.nlev; ++L) PFF_CUDA(cudaMemsetAsync(a.lv[L].cnt, 0, sizeof(int) * p.nb[L], st));
    if (weights) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int grid = std::min(div_up(N, 256), nsm * 8);
        { k_tree_seedmax<<<grid, 256, 0, st>>>(weights, N, a.status); count_launch(); }
    }
    const size_t smem = (size_t)TR_SMEM_NODES * TR_NODE_BYTES;  // per-device attribute: set on every call
    PFF_CUDA(cudaFuncSetAttribute(k_tree_level<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PFF_CUDA(cudaFuncSetAttribute(k_tree_level<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PFF_CUDA(cudaFuncSetAttribute(k_tree_level<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    PFF_PROBED("k_tree_tile<up>", st,
               k_tree_tile<false><<<p.ntiles, TR_T0_THREADS, 0, st>>>(receivers, weights, value, Q, counts, a));
    count_launch();
    for (int L = 1; L < p.nlev; ++L) {
        k_tree_level<0><<<p.nb[L], TR_LB_THREADS, smem, st>>>(L, a);
        count_launch();
    }
    { k_tree_level<2><<<1, TR_LB_THREADS, smem, st>>>(p.nlev, a); count_launch(); }
    for (int L = p.nlev - 1; L >= 1; --L) {
        k_tree_level<1><<<p.nb[L], TR_LB_THREADS, smem, st>>>(L, a);
        count_launch();
    }
    PFF_PROBED("k_tree_tile<down>", st,
               k_tree_tile<true><<<p.ntiles, TR_T0_THREADS, 0, st>>>(receivers, weights, value, Q, counts, a));
    count_launch();
    return check_cuda("pff_accumulate_tree");
}

extern "C" int pff_accumulate_tree_status(int nx, int ny, int local, void *workspace, size_t workspace_bytes,
                                          int *status, void *stream)
{
    clear_error();
    if (!status || nx < 1 || ny < 1) {
        set_error("pff_accumulate_tree_status: bad arguments");
        return PFF_ERR_ARG;
    }
    const int N = nx * ny;
    const TreePlan p = tree_plan(nx, ny, local);
    if (!workspace || workspace_bytes < tree_bytes(p, N)) {
        set_error("pff_accumulate_tree_status: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    Carver cv(workspace, workspace_bytes);
    cv.take<unsigned char>(N);
    cv.take<long long>(N);
    cv.take<unsigned>(N);
    cv.take<int>(N);
    int *stw = cv.take<int>(64);
    PFF_TRY(read_ints(IntReads().add(stw, 1), status, S(stream)));
    return PFF_OK;
}
