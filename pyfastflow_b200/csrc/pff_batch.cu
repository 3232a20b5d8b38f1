// libpff ragged batch: hundreds of independent DEM tiles of uneven sizes routed
// (receivers -> carve reroute -> accumulate) in ONE persistent launch over a packed
// layout.  Each CTA takes whole tiles from a queue (largest first) and runs the
// entire chain for its tile with block-wide barriers between passes: tiles are
// independent, so nothing synchronises across CTAs and the launch needs no host
// round trip (it can be captured in a CUDA graph).
//
// Within a tile the steps are the reference's own (pyfastflow/flow/receivers.py:31-58,
// lakeflow.py:466-538, downstream_propag.py:59-179, flowfields.py:254-292) with the
// pinned semantics of the single-grid path: serial last writer for the saddle node
// and for path reversal (largest index), the serial 2-cycle pass, serial labelling of
// receiver cycles (emulated), snapshot rake-and-compress rounds with donors in
// ascending index.  Results are bit-identical to routing each tile on its own.
#include <algorithm>
#include "pff_internal.h"

namespace pff {

struct BatchTile {
    long long off;   // first cell of the tile in the packed arrays
    long long boff;  // first basin entry (N+1 entries per tile)
    int nx, ny, mode;
    int id;          // the tile's index in the caller's order
    float dx;
    int pad;
};

// Packed per-cell and per-basin arrays of the batch (device pointers).
struct BatchArrays {
    const float *z;
    const uint8_t *codes;  // packed boundary codes of the custom-mode tiles (may be null without such tiles)
    int32_t *rcv;      // out: rerouted receivers (tile-local indices)
    float *grad;       // out: steepest gradient of the original receivers
    float *Q;          // in: per-cell seed, out: upstream sum
    uint32_t *counts;  // out: upstream cell counts
    int32_t *rec_, *rec__, *bid, *mark;
    float *zp;
    uint8_t *isb, *tag, *tag_;
    long long *saddle, *outlet;  // N+1 per tile
    int32_t *snode;              // N+1 per tile
    uint8_t *inv;                // N+1 per tile
    int32_t *dnr, *dnr_;         // 4 per cell
    int32_t *ndnr, *ndnr_, *src;
    float *p_;
    uint32_t *c_;
    const BatchTile *tiles;  // in largest-first order
    int *queue;              // [0] next tile
    int *status;             // [0] error bits (see pff_batch_status)
};

enum : int { BST_MODE = 1, BST_CYCLE_LABELS = 8, BST_CARVE = 16 };

constexpr int LB_SIDE = 32, LB_CELLS = LB_SIDE * LB_SIDE;  // label sub-blocks

struct BatchShm {
    int red;
    int cur;
    int ws[32];
    int lp[LB_CELLS];   // sub-block pointers (local indices)
    int tgt[LB_CELLS];  // sub-block cells' receivers (tile indices)
};

__device__ __forceinline__ int bceil_log2(long long n)
{
    int r = 0;
    long long p = 1;
    while (p < n) { p <<= 1; ++r; }
    return r;
}

__device__ __forceinline__ long long inv_key() { return pack_key(1e8f, 42); }

// Block-wide sum (every thread gets it).
__device__ __forceinline__ int bsum(int v, BatchShm &sh)
{
    __syncthreads();
    if (threadIdx.x == 0) sh.red = 0;
    __syncthreads();
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh.red, v);
    __syncthreads();
    const int r = sh.red;
    __syncthreads();
    return r;
}

// Block-wide exclusive prefix sum of v (blockDim a multiple of 32); *total = sum.
__device__ __forceinline__ int bscan(int v, BatchShm &sh, int *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    __syncthreads();
    if (lane == 31) sh.ws[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? sh.ws[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh.ws[lane] = s;
    }
    __syncthreads();
    const int before = (wid ? sh.ws[wid - 1] : 0) + x - v;
    *total = sh.ws[nw - 1];
    __syncthreads();
    return before;
}

#define FOR_CELLS(i, N) for (int i = threadIdx.x; i < (N); i += blockDim.x)

template <int MODE>
__device__ __forceinline__ bool leave(const Grid &g, int i)
{
    return can_leave_i<MODE>(g, i);
}

// ---- labels: basin_id_init + propagate_basin on a copy of rec_ (lakeflow.py:47-80, 507-511)
//
// Acyclic receivers: the fixed point of pointer jumping, reached in parallel.  On a
// receiver cycle the reference's serial in-place rounds give a result that depends
// only on the cycle's cells visited in ascending index; it is emulated here and every
// cell draining into the cycle takes the cycle's label.
template <int MODE>
__device__ void tile_labels(const Grid &g, int N, const int32_t *rec_, int32_t *work, int32_t *bid, int32_t *mark,
                            int32_t *scr, int rounds, BatchShm &sh, int *status)
{
    FOR_CELLS(i, N) {
        bid[i] = leave<MODE>(g, i) ? 0 : i + 1;
        work[i] = rec_[i];
        mark[i] = 0;
    }
    __syncthreads();
    for (int r = 0; r < rounds; ++r) {
        int ch = 0;
        FOR_CELLS(i, N) {
            const int p = work[i];
            const int b = bid[p], pp = work[p];
            if (bid[i] != b) { bid[i] = b; ch = 1; }
            if (pp != p) { work[i] = pp; ch = 1; }
        }
        if (!__syncthreads_or(ch)) break;
    }
    // After the rounds every pointer sits on a true root or on a cycle cell.
    int unresolved = 0;
    FOR_CELLS(i, N) {
        const int x = work[i];
        unresolved |= (rec_[x] != x);
    }
    if (!__syncthreads_or(unresolved)) return;
    // Mark every cycle cell: walkers claim cells and stop at the first cell another
    // walker claimed, which covers each cycle exactly once.
    FOR_CELLS(i, N) {
        int x = work[i];
        if (rec_[x] == x) continue;
        for (int s = 0; s <= N; ++s) {
            if (atomicExch(mark + x, 1)) break;
            x = rec_[x];
        }
    }
    __syncthreads();
    // cycle cells in ascending index order: cells[a], pos[cell] = a
    int32_t *cells = scr, *pos = scr + N, *lrec = scr + 2LL * N, *lb = scr + 3LL * N;
    int L = 0;
    for (int base = 0; base < N; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const int f = (i < N && mark[i]) ? 1 : 0;
        int tot;
        const int p = bscan(f, sh, &tot);
        if (f) { cells[L + p] = i; pos[i] = L + p; }
        L += tot;
    }
    __syncthreads();
    FOR_CELLS(a, L) {
        const int c = cells[a];
        lrec[a] = pos[rec_[c]];
        lb[a] = leave<MODE>(g, c) ? 0 : c + 1;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int r = 0; r < rounds; ++r)
            for (int a = 0; a < L; ++a) {
                lb[a] = lb[lrec[a]];
                lrec[a] = lrec[lrec[a]];
            }
    __syncthreads();
    int bad = 0;
    FOR_CELLS(a, L) bad |= (lb[a] != lb[pos[rec_[cells[a]]]]);  // one label per cycle
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, BST_CYCLE_LABELS);
    FOR_CELLS(i, N) {
        const int x = work[i];
        if (rec_[x] != x) bid[i] = lb[pos[x]];
    }
    __syncthreads();
}

// ---- labels, fast form for acyclic receivers -----------------------------------------
//
// The fixed point of the labelling is bid[i] = root(i)+1, or 0 when the root can leave.
// Roots are found in three steps: (A) each 32 x 32 sub-block is pointer-jumped in shared
// memory to its cells' terminals (an in-block root, or the last in-block cell of the
// path); J[i] = the terminal's receiver, i.e. the root itself or the entry cell of the
// next sub-block, which lies on that sub-block's perimeter; (B) pointer jumping on J over
// the perimeter cells only; (C) one gather.  A receiver cycle shows up as a pointer that
// does not settle or a final target that is not a root; the caller then runs the
// general labelling, which reproduces the serial result on cycles.
template <int MODE>
__device__ bool tile_labels_blocks(const Grid &g, int N, const int32_t *rec_, int32_t *J, int32_t *bid, BatchShm &sh)
{
    const int nx = g.nx, ny = g.ny;
    const int nbx = (nx + LB_SIDE - 1) / LB_SIDE, nby = (ny + LB_SIDE - 1) / LB_SIDE;
    int bad = 0;
    // (A) sub-block terminals
    for (int blk = 0; blk < nbx * nby; ++blk) {
        const int x0 = (blk % nbx) * LB_SIDE, y0 = (blk / nbx) * LB_SIDE;
        for (int l = threadIdx.x; l < LB_CELLS; l += blockDim.x) {
            const int x = x0 + (l & (LB_SIDE - 1)), y = y0 + l / LB_SIDE;
            int p = l, t = -1;
            if (x < nx && y < ny) {
                const int i = y * nx + x;
                t = rec_[i];
                const int ry = t / nx, rx = t - ry * nx;
                if (t != i && rx >= x0 && rx < x0 + LB_SIDE && ry >= y0 && ry < y0 + LB_SIDE)
                    p = (ry - y0) * LB_SIDE + (rx - x0);
            }
            sh.lp[l] = p;
            sh.tgt[l] = t;
        }
        __syncthreads();
        for (int r = 0; r < 10; ++r) {  // chains inside a block are shorter than 2^10 cells
            int q[LB_CELLS / 256];      // blockDim >= 256: at most 4 cells per thread
#pragma unroll
            for (int c = 0; c < LB_CELLS / 256; ++c) {
                const int l = threadIdx.x + c * blockDim.x;
                if (l < LB_CELLS) q[c] = sh.lp[sh.lp[l]];
            }
            __syncthreads();
#pragma unroll
            for (int c = 0; c < LB_CELLS / 256; ++c) {
                const int l = threadIdx.x + c * blockDim.x;
                if (l < LB_CELLS) sh.lp[l] = q[c];
            }
            __syncthreads();
        }
        for (int l = threadIdx.x; l < LB_CELLS; l += blockDim.x) {
            const int x = x0 + (l & (LB_SIDE - 1)), y = y0 + l / LB_SIDE;
            if (x >= nx || y >= ny) continue;
            const int t = sh.lp[l];
            if (sh.lp[t] != t) bad = 1;  // a cycle inside the block
            J[y * nx + x] = sh.tgt[t];
        }
        __syncthreads();
    }
    if (__syncthreads_or(bad)) return false;
    // (B) pointer jumping over the perimeter cells (every J value is a root or one of them)
    const int PER = 4 * LB_SIDE - 4;
    const int nper = nbx * nby * PER;
    bool settled = false;
    for (int r = 0; r < 64; ++r) {
        int ch = 0;
        for (int k = threadIdx.x; k < nper; k += blockDim.x) {
            const int blk = k / PER, e = k - blk * PER;
            const int x0 = (blk % nbx) * LB_SIDE, y0 = (blk / nbx) * LB_SIDE;
            const int bw = min(LB_SIDE, nx - x0), bh = min(LB_SIDE, ny - y0);  // the block's extent in the tile
            int lx, ly;  // position e on the perimeter of the bw x bh block
            if (e < LB_SIDE) { lx = e; ly = 0; }
            else if (e < 2 * LB_SIDE) { lx = e - LB_SIDE; ly = bh - 1; }
            else if (e < 3 * LB_SIDE - 2) { lx = 0; ly = e - 2 * LB_SIDE + 1; }
            else { lx = bw - 1; ly = e - (3 * LB_SIDE - 2) + 1; }
            if (lx >= bw || ly >= bh || (e >= 2 * LB_SIDE && ly >= bh - 1)) continue;
            const int x = x0 + lx, y = y0 + ly;
            const int i = y * nx + x;
            const int a = J[i], b2 = J[a];
            if (b2 != a) { J[i] = b2; ch = 1; }
        }
        if (!__syncthreads_or(ch)) { settled = true; break; }
    }
    if (!settled) return false;
    // (C) gather, and check that every target is a true root
    FOR_CELLS(i, N) {
        int t = J[i];
        if (rec_[t] != t) t = J[t];
        if (rec_[t] != t) { bad = 1; continue; }
        bid[i] = leave<MODE>(g, t) ? 0 : t + 1;
    }
    return !__syncthreads_or(bad);
}

// ---- saddlesort passes 1-5 (lakeflow.py:106-281) ------------------------------------
template <int MODE>
__device__ void tile_saddlesort(const Grid &g, int N, const int32_t *bid, uint8_t *isb, float *zp, long long *sad,
                                int32_t *snode, long long *out, uint8_t *inv, const float *z, const int32_t *pl,
                                int np)
{
    // With labels of acyclic receivers (pl given) the only basin ids are 0 and pit + 1 for
    // the current pits (pl, np entries): those entries are reset and the per-basin passes
    // run over the pit list.  Otherwise (labels of a receiver cycle, pl == nullptr) every
    // basin id 0..N is reset and scanned, as in the reference.  Basin N is skipped by the
    // per-basin passes, as the reference's loops over b < N skip it.
    const long long iv = inv_key();
    const int ninit = pl ? np + 1 : N + 1, nscan = pl ? np : N;
    for (int k = threadIdx.x; k < ninit; k += blockDim.x) {
        const int b = pl ? (k < np ? pl[k] + 1 : 0) : k;
        sad[b] = iv;
        out[b] = iv;
        snode[b] = -1;
        inv[b] = 0;
    }
    __syncthreads();
    // passes 1 and 2: z' and the per-basin lowest packed (z', neighbour basin)
    FOR_CELLS(i, N) {
        const float zi = z[i];
        if (leave<MODE>(g, i)) {
            zp[i] = zi;
            isb[i] = 0;  // never written by the reference: its zero initial value
            continue;
        }
        const int row = i / g.nx, col = i - row * g.nx;
        const int bi = bid[i];
        int js[4];
        neighbours4<MODE>(g, i, row, col, js);
        bool border = false;
        float zn = 1e9f;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (js[k] != -1 && bid[js[k]] != bi) {
                border = true;
                zn = fminf(zn, z[js[k]]);
            }
        isb[i] = border;
        const float zpi = border ? fmaxf(zi, zn) : 1e9f;
        zp[i] = zpi;
        if (!border) continue;
        long long res = iv;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (js[k] == -1) continue;
            const int bj = bid[js[k]];
            if (bj != bi) {
                const long long c = pack_key(zpi, bj);
                res = c < res ? c : res;
            }
        }
        if (res != iv) atomicMin(sad + bi, res);
    }
    __syncthreads();
    // pass 3: saddle node = largest qualifying index (serial last writer)
    FOR_CELLS(i, N) {
        if (!isb[i]) continue;
        const int bi = bid[i];
        if (bi == 0) continue;
        const long long s = sad[bi];
        const float tz = key_value(s);
        const int tb = key_index(s);
        const float zpi = zp[i];
        const int row = i / g.nx, col = i - row * g.nx;
        int js[4];
        neighbours4<MODE>(g, i, row, col, js);
        bool here = false;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (js[k] != -1 && bid[js[k]] == tb && zpi == tz) here = true;
        if (here) atomicMax(snode + bi, i);
    }
    __syncthreads();
    // pass 4: outlet = lowest foreign neighbour of the saddle node (first k wins)
    for (int k0 = threadIdx.x; k0 < nscan; k0 += blockDim.x) {
        const int b = pl ? pl[k0] + 1 : k0;
        if (b == 0 || b >= N || sad[b] == iv) continue;
        const int node = snode[b];
        if (node < 0) continue;
        float tz = 1e9f;
        int r = -1;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = neighbour_i<MODE>(g, node, k);
            if (j == -1) continue;
            const float zj = z[j];
            if (bid[j] != b && tz > zj) {
                tz = zj;
                r = j;
            }
        }
        if (r > -1) out[b] = pack_key(tz, r);
    }
    __syncthreads();
    // pass 5: 2-cycles b -> b' -> b with b' < b, snapshot reads, plus the one basin
    // (bid[42]) whose serial outcome can differ from the snapshot
    for (int k0 = threadIdx.x; k0 < nscan; k0 += blockDim.x) {
        const int b = pl ? pl[k0] + 1 : k0;
        if (b == 0 || b >= N) continue;
        const long long ob = out[b];
        if (ob == iv) continue;
        const int bd1 = bid[key_index(ob)];
        if (bd1 == 0) continue;
        const int ro2 = key_index(out[bd1]);
        const int bd2 = (ro2 >= 0 && ro2 < N) ? bid[ro2] : -1;
        if (bd2 == b && bd1 < b) inv[b] = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0 && N > 42) {
        const int D = bid[42];
        if (D > 0 && D < N && out[D] != iv) {
            const int bd1 = bid[key_index(out[D])];
            if (bd1 != 0 && bd1 < D && inv[bd1]) inv[D] = 1;
        }
    }
    __syncthreads();
    for (int k0 = threadIdx.x; k0 < nscan; k0 += blockDim.x) {
        const int b = pl ? pl[k0] + 1 : k0;
        if (b < N && inv[b]) {
            out[b] = iv;
            sad[b] = iv;
            snode[b] = -1;
        }
    }
    __syncthreads();
}

// ---- reroute_carve (lakeflow.py:308-438); leaves the result in rec and rec_ ----------
//
// The reference tags the saddle nodes and propagates the tags by pointer jumping until
// no tag changes; a round adds the next 2^r cells of every tagged path, so the fixed
// point is the union of the saddle nodes' forward orbits under rec_ (down to each
// pit, or around a receiver cycle).  The jumped pointers are discarded by the
// finalisation, so only that tag set matters: here each saddle node walks its own
// orbit, stopping at a cell already tagged (the rest of that orbit is another
// walker's) or at a root.
__device__ void tile_carve(int N, int32_t *rec, int32_t *rec_, int32_t *claim, uint8_t *tag, const int32_t *snode,
                           const long long *out, const int32_t *pl, int np, int *status)
{
    const long long iv = inv_key();
    FOR_CELLS(i, N) {
        tag[i] = 0;
        claim[i] = -1;
    }
    __syncthreads();
    int overrun = 0;
    const int nscan = pl ? np : N;  // the pits' basins, or every basin id (see tile_saddlesort)
    for (int k0 = threadIdx.x; k0 < nscan; k0 += blockDim.x) {
        const int b = pl ? pl[k0] + 1 : k0;
        if (b >= N) continue;
        int x = snode[b];
        if (x == -1) continue;
        int s = 0;
        for (; s <= N; ++s) {
            if (tag[x]) break;
            tag[x] = 1;
            const int nx_ = rec_[x];
            if (nx_ == x) break;
            x = nx_;
        }
        if (s > N) overrun = 1;
    }
    if (__syncthreads_or(overrun) && threadIdx.x == 0) atomicOr(status, BST_CARVE);
    // finalise: pre-carve receivers, path reversal (largest index wins), saddle links
    FOR_CELLS(i, N) {
        const int r0 = rec_[i];
        rec[i] = r0;
        if (tag[r0] && tag[i] && i != r0) atomicMax(claim + r0, i);
    }
    __syncthreads();
    FOR_CELLS(x, N) {
        const int c = claim[x];
        if (c >= 0) rec[x] = c;
    }
    __syncthreads();
    for (int k0 = threadIdx.x; k0 < nscan; k0 += blockDim.x) {
        const int b = pl ? pl[k0] + 1 : k0;
        if (b >= N) continue;
        const long long ob = out[b];
        if (ob != iv) rec[snode[b]] = key_index(ob);
    }
    __syncthreads();
    FOR_CELLS(i, N) rec_[i] = rec[i];
    __syncthreads();
}

// ---- rake-and-compress (downstream_propag.py:21-179), f32 and u32 payloads ---------------
__device__ __forceinline__ bool bget_src(const int32_t *src, int t, int it)
{
    const int e = src[t];
    bool flip = e < 0;
    if (abs(e) == it + 1) flip = !flip;
    return flip;
}

// Only nodes that still have donors are visited: a node with none left does nothing
// in any later round, so the rounds run over a compacted active list (la -> lb).
__device__ void tile_accumulate(int N, const int32_t *rcv, float *p, uint32_t *c, int32_t *dnr, int32_t *dnr_,
                                int32_t *ndnr, int32_t *ndnr_, int32_t *src, float *p_, uint32_t *c_, int32_t *la,
                                int32_t *lb, BatchShm &sh)
{
    FOR_CELLS(t, N) {
        ndnr[t] = 0;
        src[t] = 0;
        c[t] = 1u;
    }
    __syncthreads();
    FOR_CELLS(t, N) {  // rcv2donor (:78-96); D4 receivers give at most 4 donors
        const int r = rcv[t];
        if (r == t) continue;
        const int slot = atomicAdd(ndnr + r, 1);
        if (slot < 4) dnr[4LL * r + slot] = t;
    }
    __syncthreads();
    int nact = 0;
    for (int b0 = 0; b0 < N; b0 += blockDim.x) {  // sort donors (ascending: the serial slot order), list actives
        const int r = b0 + threadIdx.x;
        int f = 0;
        if (r < N) {
            const int n = min(ndnr[r], 4);
            int *d = dnr + 4LL * r;
            for (int a = 1; a < n; ++a) {
                const int x = d[a];
                int b = a - 1;
                while (b >= 0 && d[b] > x) {
                    d[b + 1] = d[b];
                    --b;
                }
                d[b + 1] = x;
            }
            f = n > 0;
        }
        int tot;
        const int q = bscan(f, sh, &tot);
        if (f) la[nact + q] = r;
        nact += tot;
    }
    __syncthreads();
    const int logn = bceil_log2(N) + 1;
    for (int it = 0; it <= logn && nact > 0; ++it) {
        int worked_any = 0, nnext = 0;
        for (int b0 = 0; b0 < nact; b0 += blockDim.x) {
            const int k = b0 + threadIdx.x;
            int keep = 0, tid = -1;
            if (k < nact) {
                tid = la[k];
                const bool flip = bget_src(src, tid, it);
                int todo = flip ? ndnr_[tid] : ndnr[tid];
                const long long base = 4LL * tid;
                int donors[4] = {-1, -1, -1, -1};
                bool worked = false;
                float padd = 0.f;
                uint32_t cadd = 0;
                int i = 0;
                while (i < todo && i < 4) {
                    if (donors[i] == -1) donors[i] = flip ? dnr_[base + i] : dnr[base + i];
                    const int did = donors[i];
                    const bool fd = bget_src(src, did, it);
                    const int nd = fd ? ndnr_[did] : ndnr[did];
                    if (nd <= 1) {
                        if (!worked) {
                            padd = flip ? p_[tid] : p[tid];
                            cadd = flip ? c_[tid] : c[tid];
                        }
                        worked = true;
                        padd = __fadd_rn(padd, fd ? p_[did] : p[did]);
                        cadd += fd ? c_[did] : c[did];
                        if (nd == 0) {
                            --todo;
                            if (todo > i) donors[i] = flip ? dnr_[base + todo] : dnr[base + todo];
                            --i;
                        } else {
                            donors[i] = fd ? dnr_[4LL * did] : dnr[4LL * did];
                        }
                    }
                    ++i;
                }
                if (worked) {
                    worked_any = 1;
                    const int m = todo < 4 ? todo : 4;
                    if (flip) {
                        ndnr[tid] = todo;
                        p[tid] = padd;
                        c[tid] = cadd;
                        for (int j = 0; j < m; ++j) dnr[base + j] = donors[j];
                    } else {
                        ndnr_[tid] = todo;
                        p_[tid] = padd;
                        c_[tid] = cadd;
                        for (int j = 0; j < m; ++j) dnr_[base + j] = donors[j];
                    }
                    src[tid] = (flip ? 1 : -1) * (it + 1);
                }
                keep = todo > 0;
            }
            int tot;
            const int q = bscan(keep, sh, &tot);
            if (keep) lb[nnext + q] = tid;
            nnext += tot;
        }
        // a round in which nothing worked leaves the state, and every later round, unchanged
        if (!__syncthreads_or(worked_any)) break;
        int32_t *t = la;
        la = lb;
        lb = t;
        nact = nnext;
    }
    FOR_CELLS(t, N) {  // fuse(Q, src, Q_, logn)
        if (bget_src(src, t, logn)) {
            p[t] = p_[t];
            c[t] = c_[t];
        }
    }
    __syncthreads();
}

// receivers (receivers.py:31-58): strict >, first k wins ties.  Writes rec and rec_
// (and the gradient if grad is not null).
template <int MODE>
__device__ void tile_receivers(const Grid &g, float dx, const float *z, int32_t *rec, int32_t *rec_, float *grad)
{
    const int N = g.nx * g.ny;
    FOR_CELLS(i, N) {
        const int row = i / g.nx, col = i - row * g.nx;
        int js[4];
        neighbours4<MODE>(g, i, row, col, js);
        const float zi = z[i];
        int r = i;
        float sr = 0.f, dbest = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (js[k] == -1) continue;
            const float d = __fsub_rn(zi, z[js[k]]);
            if (d > dbest) {  // a smaller difference cannot give a larger quotient
                const float q = __fdiv_rn(d, dx);
                if (q > sr) {
                    sr = q;
                    r = js[k];
                    dbest = d;
                }
            }
        }
        rec[i] = r;
        rec_[i] = r;
        if (grad) grad[i] = sr;
    }
    __syncthreads();
}

// reroute_flow(carve=True) (lakeflow.py:466-538) on receivers rec (with rec_ == rec).
template <int MODE>
__device__ void tile_reroute(const Grid &g, const BatchTile &T, const BatchArrays &A, const float *z, BatchShm &sh)
{
    const int N = g.nx * g.ny;
    const long long o = T.off, ob = T.boff;
    int32_t *rec = A.rcv + o, *rec_ = A.rec_ + o, *rec__ = A.rec__ + o, *bid = A.bid + o;
    const int lrounds = bceil_log2(N) + 1;
    int32_t *pl = A.ndnr + o;  // pit list (scratch of the accumulation / diffusion, free here)
    auto list_pits = [&]() {   // depression_counter (lakeflow.py:25-44), as an ascending list
        int n = 0;
        for (int b0 = 0; b0 < N; b0 += blockDim.x) {
            const int i = b0 + threadIdx.x;
            const int f = (i < N && rec_[i] == i && !leave<MODE>(g, i)) ? 1 : 0;
            int tot;
            const int q = bscan(f, sh, &tot);
            if (f) pl[n + q] = i;
            n += tot;
        }
        __syncthreads();
        return n;
    };
    const int ndep = list_pits();
    if (ndep == 0) return;
    const int outer = bceil_log2(ndep) + 1;
    for (int it = 0; it < outer; ++it) {
        const int nd = it > 0 ? list_pits() : ndep;
        if (nd == 0) break;  // (the labels the reference computes first are overwritten)
        const bool acyclic = tile_labels_blocks<MODE>(g, N, rec_, rec__, bid, sh);
        if (!acyclic) tile_labels<MODE>(g, N, rec_, rec__, bid, A.mark + o, A.dnr + 4 * o, lrounds, sh, A.status);
        const int32_t *bl = acyclic ? pl : nullptr;  // basin ids: the pits', or any (labels of a cycle)
        tile_saddlesort<MODE>(g, N, bid, A.isb + o, A.zp + o, A.saddle + ob, A.snode + ob, A.outlet + ob,
                              A.inv + ob, z, bl, nd);
        tile_carve(N, rec, rec_, A.mark + o, A.tag + o, A.snode + ob, A.outlet + ob, bl, nd, A.status);
    }
}

template <int MODE>
__device__ void route_tile(const BatchTile &T, const BatchArrays &A, BatchShm &sh)
{
    const Grid g{T.nx, T.ny, MODE, MODE == 3 ? A.codes + T.off : nullptr};
    const int N = T.nx * T.ny;
    const long long o = T.off;
    const float *z = A.z + o;
    tile_receivers<MODE>(g, T.dx, z, A.rcv + o, A.rec_ + o, A.grad + o);
    tile_reroute<MODE>(g, T, A, z, sh);
    // accumulate: Q holds the seed (flowfields.py:272-292)
    tile_accumulate(N, A.rcv + o, A.Q + o, A.counts + o, A.dnr + 4 * o, A.dnr_ + 4 * o, A.ndnr + o, A.ndnr_ + o,
                    A.src + o, A.p_ + o, A.c_ + o, A.mark + o, A.rec__ + o, sh);
}

// ---- GraphFlood on a tile (gf_fields.py:126-141) --------------------------------------
//
// One iteration: receivers, carve reroute, fill with delta (fill_topo.py:17-45,
// snapshot rounds), 5 diffusion sweeps (gf_hydrodynamics.py:24-75, sums in the
// serial order), Manning update (gf_hydrodynamics.py:79-129).  Per-tile constants
// are the f32 values the single-grid Flooder passes: dx2, prec*dx^2, manning.
struct GfParams {
    const float *cst;  // per tile (caller order): dx2, prec_dx2, manning, stop threshold on max|dh|
    float edgesw, dt, eps;
    int niter;
    int crit;          // 0: stop when max|dh| < threshold; 1: when mean|dh| < threshold; -1: never
    float *h;          // packed, in/out
    int32_t *iters;    // per tile (caller order): iterations run
    float *res;        // per tile: last max|dh| and mean|dh| (2 floats)
    float *trace;      // optional, per tile: niter x (max|dh|, mean|dh|)
};

// max and sum of v over the block (max as unsigned bits: |x| >= 0, NaN above all)
__device__ __forceinline__ void bmaxsum(float m, float sum, BatchShm &sh, float *om, float *os)
{
    unsigned mu = __float_as_uint(m);
    for (int o = 16; o; o >>= 1) {
        mu = max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
    }
    __syncthreads();
    if (threadIdx.x == 0) { sh.ws[0] = 0; sh.ws[1] = 0; }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        atomicMax((unsigned *)&sh.ws[0], mu);
        atomicAdd((float *)&sh.ws[1], sum);
    }
    __syncthreads();
    *om = __uint_as_float((unsigned)sh.ws[0]);
    *os = __int_as_float(sh.ws[1]);
    __syncthreads();
}

template <int MODE>
__device__ void gf_tile(const BatchTile &T, const BatchArrays &A, const GfParams &P, BatchShm &sh)
{
    const Grid g{T.nx, T.ny, MODE, MODE == 3 ? A.codes + T.off : nullptr};
    const int N = T.nx * T.ny;
    const long long o = T.off;
    float *zh = const_cast<float *>(A.z) + o, *h = P.h + o, *Q = A.Q + o;
    int32_t *rec = A.rcv + o;
    // scratch of the routing arrays, free once the reroute is done
    int32_t *ra = A.rec_ + o, *rb = A.rec__ + o;
    float *zs = A.zp + o, *zn = A.p_ + o;
    float *w = reinterpret_cast<float *>(A.dnr_) + 4 * o;
    uint8_t *issrc = A.isb + o;
    float *temp = reinterpret_cast<float *>(A.ndnr) + o;
    float *href = reinterpret_cast<float *>(A.c_) + o;
    float *dh = reinterpret_cast<float *>(A.ndnr_) + o;
    const float dx = T.dx, dx2 = P.cst[4 * T.id], prec_dx2 = P.cst[4 * T.id + 1], manning = P.cst[4 * T.id + 2];
    const float thr = P.cst[4 * T.id + 3];
    const int nr = bceil_log2(N);
    int it = 0;
    float rmax = 0.f, rmean = 0.f;
    for (; it < P.niter; ++it) {
        FOR_CELLS(i, N) href[i] = h[i];
        tile_receivers<MODE>(g, dx, zh, rec, A.rec_ + o, nullptr);
        tile_reroute<MODE>(g, T, A, zh, sh);
        // fill_z_add_delta (fill_topo.py:99-125): rounds on snapshots of z_ and rec_
        FOR_CELLS(i, N) {
            zs[i] = zh[i];
            ra[i] = rec[i];
        }
        __syncthreads();
        float *a = zs, *b = zn;
        int32_t *pa = ra, *pb = rb;
        for (int r = 0; r < nr; ++r) {
            const float inc = (float)(ldexp(1.0, r - 1) * (double)P.eps);
            int ch = 0;
            FOR_CELLS(i, N) {
                const int q = pa[i];
                const int qq = pa[q];
                pb[i] = qq;
                const float zi = a[i];
                float zo = zi;
                if (!(i == q || (zi > zh[q] && qq == q))) zo = fmaxf(zi, __fadd_rn(a[q], inc));
                b[i] = zo;
                ch |= qq != q || __float_as_uint(zo) != __float_as_uint(zi);
            }
            const bool any = __syncthreads_or(ch);
            float *t = a; a = b; b = t;
            int32_t *u = pa; pa = pb; pb = u;
            // a round that changed nothing is a fixed point of every later round (see k_fill_round)
            if (!any) break;
        }
        FOR_CELLS(i, N) {
            const float zf = a[i];
            h[i] = __fadd_rn(h[i], __fsub_rn(zf, zh[i]));
            zh[i] = zf;
        }
        __syncthreads();
        // diffusion: weights once, then 5 gather sweeps (Q <-> temp), ending in Q
        FOR_CELLS(i, N) {
            const int row = i / g.nx, col = i - row * g.nx;
            if (leave<MODE>(g, i)) { issrc[i] = 0; continue; }
            const float zi = zh[i];
            float sk[4];
            float sums = 0.f;
            int js[4];
            neighbours4<MODE>(g, i, row, col, js);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                sk[k] = (js[k] != -1) ? fmaxf(0.f, __fdiv_rn(__fsub_rn(zi, zh[js[k]]), dx)) : 0.f;
                sums = __fadd_rn(sums, sk[k]);
            }
            if (sums == 0.f) { issrc[i] = 0; continue; }
            issrc[i] = 1;
#pragma unroll
            for (int k = 0; k < 4; ++k) w[(size_t)k * N + i] = __fdiv_rn(sk[k], sums);
        }
        __syncthreads();
        float *qa = Q, *qb = temp;
        for (int sw = 0; sw < 5; ++sw) {
            FOR_CELLS(j, N) {
                const int row = j / g.nx, col = j - row * g.nx;
                float acc = prec_dx2;
                if (MODE != 3 && row > 0 && row < g.ny - 1 && col > 0 && col < g.nx - 1) {
                    const int nx = g.nx;
                    if (issrc[j - nx]) acc = __fadd_rn(acc, __fmul_rn(w[3 * (size_t)N + j - nx], qa[j - nx]));
                    if (issrc[j - 1]) acc = __fadd_rn(acc, __fmul_rn(w[2 * (size_t)N + j - 1], qa[j - 1]));
                    if (issrc[j + 1]) acc = __fadd_rn(acc, __fmul_rn(w[(size_t)N + j + 1], qa[j + 1]));
                    if (issrc[j + nx]) acc = __fadd_rn(acc, __fmul_rn(w[j + nx], qa[j + nx]));
                } else {
                    int c[8];
                    const int n = donor_candidates(g, j, row, col, c);
                    for (int q = 0; q < n; ++q) {
                        const int i = c[q];
                        if (!issrc[i]) continue;
                        const float qi = qa[i];
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (neighbour_i<MODE>(g, i, k) == j) acc = __fadd_rn(acc, __fmul_rn(w[(size_t)k * N + i], qi));
                    }
                }
                qb[j] = acc;
            }
            __syncthreads();
            float *t = qa; qa = qb; qb = t;
        }
        if (qa != Q) {
            FOR_CELLS(j, N) Q[j] = qa[j];
            __syncthreads();
        }
        // Manning update, two loops as in the reference (h receives tdh twice)
        FOR_CELLS(i, N) {
            const int r = rec[i];
            float tS = P.edgesw;
            if (r != i) tS = fmaxf(__fdiv_rn(__fsub_rn(zh[i], zh[r]), dx), 1e-4f);
            float Qo = __fmul_rn(dx, (float)pow((double)h[i], (double)(5.0f / 3.0f)));
            Qo = __fdiv_rn(Qo, manning);
            Qo = __fmul_rn(Qo, __fsqrt_rn(tS));
            float tdh = __fdiv_rn(__fsub_rn(Q[i], Qo), dx2);
            tdh = __fmul_rn(tdh, P.dt);
            const float h1 = __fadd_rn(h[i], tdh);
            h[i] = h1;
            if (h1 < 0.f) tdh = __fadd_rn(tdh, h1);
            dh[i] = tdh;
        }
        __syncthreads();
        float m = 0.f, sum = 0.f;
        FOR_CELLS(i, N) {
            const float d = dh[i];
            const float hn = __fadd_rn(h[i], d);
            h[i] = hn;
            zh[i] = __fadd_rn(zh[i], d);
            const float e = fabsf(__fsub_rn(hn, href[i]));
            m = __uint_as_float(max(__float_as_uint(m), __float_as_uint(e)));
            sum += e;
        }
        bmaxsum(m, sum, sh, &rmax, &rmean);
        rmean /= (float)N;
        if (P.trace && threadIdx.x == 0) {
            P.trace[((size_t)T.id * P.niter + it) * 2] = rmax;
            P.trace[((size_t)T.id * P.niter + it) * 2 + 1] = rmean;
        }
        if ((P.crit == 0 && rmax < thr) || (P.crit == 1 && rmean < thr)) { ++it; break; }
    }
    if (threadIdx.x == 0) {
        P.iters[T.id] = it;
        P.res[2 * T.id] = rmax;
        P.res[2 * T.id + 1] = rmean;
    }
    __syncthreads();
}

// Persistent: each CTA takes the next tile (largest first) until the queue is empty.
__global__ void __launch_bounds__(1024) k_batch_route(int ntiles, BatchArrays A)
{
    __shared__ BatchShm sh;
    for (;;) {
        if (threadIdx.x == 0) sh.cur = atomicAdd(A.queue, 1);
        __syncthreads();
        const int k = sh.cur;
        __syncthreads();
        if (k >= ntiles) return;
        const BatchTile T = A.tiles[k];
        switch (T.mode) {
        case 0: route_tile<0>(T, A, sh); break;
        case 1: route_tile<1>(T, A, sh); break;
        case 2: route_tile<2>(T, A, sh); break;
        case 3:
            if (A.codes) route_tile<3>(T, A, sh);
            else if (threadIdx.x == 0) atomicOr(A.status, BST_MODE);
            break;
        default:
            if (threadIdx.x == 0) atomicOr(A.status, BST_MODE);
            break;
        }
        __syncthreads();
    }
}

// Persistent GraphFlood: each CTA runs whole tiles to their stop, largest first.
__global__ void __launch_bounds__(1024) k_batch_graphflood(int ntiles, BatchArrays A, GfParams P)
{
    __shared__ BatchShm sh;
    for (;;) {
        if (threadIdx.x == 0) sh.cur = atomicAdd(A.queue, 1);
        __syncthreads();
        const int k = sh.cur;
        __syncthreads();
        if (k >= ntiles) return;
        const BatchTile T = A.tiles[k];
        switch (T.mode) {
        case 0: gf_tile<0>(T, A, P, sh); break;
        case 1: gf_tile<1>(T, A, P, sh); break;
        case 2: gf_tile<2>(T, A, P, sh); break;
        case 3:
            if (A.codes) gf_tile<3>(T, A, P, sh);
            else if (threadIdx.x == 0) atomicOr(A.status, BST_MODE);
            break;
        default:
            if (threadIdx.x == 0) atomicOr(A.status, BST_MODE);
            break;
        }
        __syncthreads();
    }
}

__global__ void k_batch_reset(int *ctr)
{
    ctr[0] = 0;
    ctr[1] = 0;
}

// Workspace layout, identical for the plan and the launches.
struct BatchWs {
    BatchArrays A;
    BatchTile *tiles;
    int *ctr;
    bool ok;
};

static BatchWs carve_batch(void *ws, size_t wsb, long long total, int ntiles)
{
    Carver cv(ws, wsb);
    const size_t n = (size_t)total, nb = n + (size_t)ntiles;
    BatchWs w{};
    BatchArrays &A = w.A;
    w.ctr = cv.take<int>(64);
    w.tiles = cv.take<BatchTile>((size_t)ntiles);
    A.rec_ = cv.take<int32_t>(n);
    A.rec__ = cv.take<int32_t>(n);
    A.bid = cv.take<int32_t>(n);
    A.mark = cv.take<int32_t>(n);
    A.zp = cv.take<float>(n);
    A.isb = cv.take<uint8_t>(n);
    A.tag = cv.take<uint8_t>(n);
    A.tag_ = cv.take<uint8_t>(n);
    A.saddle = cv.take<long long>(nb);
    A.outlet = cv.take<long long>(nb);
    A.snode = cv.take<int32_t>(nb);
    A.inv = cv.take<uint8_t>(nb);
    A.dnr = cv.take<int32_t>(4 * n);
    A.dnr_ = cv.take<int32_t>(4 * n);
    A.ndnr = cv.take<int32_t>(n);
    A.ndnr_ = cv.take<int32_t>(n);
    A.src = cv.take<int32_t>(n);
    A.p_ = cv.take<float>(n);
    A.c_ = cv.take<uint32_t>(n);
    A.tiles = w.tiles;
    A.queue = w.ctr;
    A.status = w.ctr + 1;
    w.ok = A.c_ != nullptr;
    return w;
}

}  // namespace pff

using namespace pff;

extern "C" size_t pff_batch_workspace_bytes(long long total_cells, int ntiles)
{
    if (total_cells <= 0 || ntiles <= 0) return 0;
    const size_t n = (size_t)total_cells, nb = n + (size_t)ntiles;
    return Carver::round(64 * 4) + Carver::round(sizeof(BatchTile) * (size_t)ntiles) + Carver::round(4 * n) * 5 +
           Carver::round(n) * 3 + Carver::round(8 * nb) * 2 + Carver::round(4 * nb) + Carver::round(nb) +
           Carver::round(16 * n) * 2 + Carver::round(4 * n) * 5 + 256;
}

namespace pff {
static int batch_check(long long total, int ntiles, void *ws, size_t wsb, const char *who)
{
    if (ntiles <= 0 || total <= 0) {
        set_error("%s: empty batch", who);
        return PFF_ERR_ARG;
    }
    if (!ws || wsb < pff_batch_workspace_bytes(total, ntiles)) {
        set_error("%s: workspace too small", who);
        return PFF_ERR_WORKSPACE;
    }
    return PFF_OK;
}
}  // namespace pff

extern "C" long long pff_batch_plan(const int32_t *tile_nx, const int32_t *tile_ny, const int32_t *tile_mode,
                                    const float *tile_dx, int ntiles, long long *tile_offset, int32_t *order,
                                    void *workspace, size_t workspace_bytes, void *stream)
{
    clear_error();
    if (ntiles <= 0 || !tile_nx || !tile_ny || !tile_mode || !tile_dx || !tile_offset) {
        set_error("pff_batch_plan: bad arguments");
        return -PFF_ERR_ARG;
    }
    long long off = 0;
    for (int t = 0; t < ntiles; ++t) {
        const int nx = tile_nx[t], ny = tile_ny[t], md = tile_mode[t];
        if (nx < 2 || ny < 2 || md < 0 || md > 3 || (long long)nx * ny * 4 >= (1LL << 31) ||
            !(tile_dx[t] > 0.f)) {
            set_error("pff_batch_plan: tile %d: bad size %dx%d, mode %d or dx (modes 0-3)", t, nx, ny,
                      md);
            return -PFF_ERR_ARG;
        }
        tile_offset[t] = off;
        off += (long long)nx * ny;
    }
    const long long total = off;
    if (!workspace) return total;  // size query
    const int rc = batch_check(total, ntiles, workspace, workspace_bytes, "pff_batch_plan");
    if (rc) return -rc;
    // largest tiles first (longest-processing-time order); equal sizes by tile index
    int *ord = new int[ntiles];
    for (int t = 0; t < ntiles; ++t) ord[t] = t;
    auto cells = [&](int t) { return (long long)tile_nx[t] * tile_ny[t]; };
    std::stable_sort(ord, ord + ntiles, [&](int a, int b) { return cells(a) > cells(b); });
    BatchTile *ht = new BatchTile[ntiles];
    for (int k = 0; k < ntiles; ++k) {
        const int t = ord[k];
        ht[k] = BatchTile{tile_offset[t], tile_offset[t] + t, tile_nx[t], tile_ny[t], tile_mode[t], t, tile_dx[t], 0};
        if (order) order[k] = t;
    }
    BatchWs w = carve_batch(workspace, workspace_bytes, total, ntiles);
    cudaStream_t st = S(stream);
    const cudaError_t e1 = cudaMemcpyAsync(w.tiles, ht, sizeof(BatchTile) * ntiles, cudaMemcpyHostToDevice, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);  // the host array must outlive the copy
    delete[] ht;
    delete[] ord;
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        set_error("pff_batch_plan: descriptor upload: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
        return -PFF_ERR_CUDA;
    }
    return total;
}

extern "C" int pff_batch_route(const float *z, const uint8_t *codes, int32_t *receivers, float *gradient, float *Q,
                               uint32_t *counts, long long total_cells, int ntiles, int threads, int ctas_per_sm,
                               void *workspace, size_t workspace_bytes, void *stream)
{
    clear_error();
    PFF_TRY(batch_check(total_cells, ntiles, workspace, workspace_bytes, "pff_batch_route"));
    if (!z || !receivers || !gradient || !Q || !counts) {
        set_error("pff_batch_route: null pointer");
        return PFF_ERR_ARG;
    }
    if (threads != 256 && threads != 512 && threads != 1024) {
        set_error("pff_batch_route: threads must be 256, 512 or 1024 (got %d)", threads);
        return PFF_ERR_ARG;
    }
    int dev = 0, nsm = 148, occ = 1;
    PFF_CUDA(cudaGetDevice(&dev));
    PFF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PFF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_route, threads, 0));
    if (ctas_per_sm < 1) ctas_per_sm = 1;
    if (ctas_per_sm > occ) ctas_per_sm = occ > 0 ? occ : 1;
    BatchWs w = carve_batch(workspace, workspace_bytes, total_cells, ntiles);
    BatchArrays A = w.A;
    A.z = z;
    A.codes = codes;
    A.rcv = receivers;
    A.grad = gradient;
    A.Q = Q;
    A.counts = counts;
    cudaStream_t st = S(stream);
    const int grid = std::min(nsm * ctas_per_sm, ntiles);
    { k_batch_reset<<<1, 1, 0, st>>>(w.ctr); count_launch(); }
    { k_batch_route<<<grid, threads, 0, st>>>(ntiles, A); count_launch(); }
    return check_cuda("pff_batch_route");
}

extern "C" int pff_batch_status(long long total_cells, int ntiles, void *workspace, size_t workspace_bytes,
                                int *status, void *stream)
{
    clear_error();
    PFF_TRY(batch_check(total_cells, ntiles, workspace, workspace_bytes, "pff_batch_status"));
    if (!status) {
        set_error("pff_batch_status: null pointer");
        return PFF_ERR_ARG;
    }
    BatchWs w = carve_batch(workspace, workspace_bytes, total_cells, ntiles);
    cudaStream_t st = S(stream);
    PFF_CUDA(cudaMemcpyAsync(status, w.A.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    PFF_CUDA(cudaStreamSynchronize(st));
    return PFF_OK;
}

extern "C" int pff_batch_graphflood(float *zh, const uint8_t *codes, float *h, float *Q, const float *tile_consts,
                                    float edgesw, float dt,
                                    int niter, int crit, int32_t *iters, float *residuals, float *trace,
                                    long long total_cells, int ntiles, int threads, int ctas_per_sm, void *workspace,
                                    size_t workspace_bytes, void *stream)
{
    clear_error();
    PFF_TRY(batch_check(total_cells, ntiles, workspace, workspace_bytes, "pff_batch_graphflood"));
    if (!zh || !h || !Q || !tile_consts || !iters || !residuals || niter < 0 || crit < -1 || crit > 1) {
        set_error("pff_batch_graphflood: bad arguments");
        return PFF_ERR_ARG;
    }
    if (threads != 256 && threads != 512 && threads != 1024) {
        set_error("pff_batch_graphflood: threads must be 256, 512 or 1024 (got %d)", threads);
        return PFF_ERR_ARG;
    }
    int dev = 0, nsm = 148, occ = 1;
    PFF_CUDA(cudaGetDevice(&dev));
    PFF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    PFF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_graphflood, threads, 0));
    if (ctas_per_sm < 1) ctas_per_sm = 1;
    if (ctas_per_sm > occ) ctas_per_sm = occ > 0 ? occ : 1;
    BatchWs w = carve_batch(workspace, workspace_bytes, total_cells, ntiles);
    BatchArrays A = w.A;
    A.z = zh;
    A.codes = codes;
    A.Q = Q;
    A.rcv = A.src;  // the rerouted receivers of each iteration (the accumulation arrays are unused)
    A.grad = nullptr;
    A.counts = nullptr;
    GfParams P{tile_consts, edgesw, dt, 1e-3f, niter, crit, h, iters, residuals, trace};
    cudaStream_t st = S(stream);
    const int grid = std::min(nsm * ctas_per_sm, ntiles);
    { k_batch_reset<<<1, 1, 0, st>>>(w.ctr); count_launch(); }
    { k_batch_graphflood<<<grid, threads, 0, st>>>(ntiles, A, P); count_launch(); }
    return check_cuda("pff_batch_graphflood");
}
