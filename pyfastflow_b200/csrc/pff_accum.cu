// libpff accumulation: donor inversion and rake-and-compress tree contraction.
//
// Semantics follow pyfastflow/flow/downstream_propag.py exactly:
//   - donor slots hold donors in ascending cell index (the reference's serial
//     atomic order, :88-96);
//   - each round reads a consistent start-of-round snapshot through the
//     ping-pong buffers and per-node epoch tags src = +-(round+1) (:21-56), so
//     the result is independent of thread scheduling and bit-identical to the
//     serial execution, f32 sums included.
// The structure of the contraction (which donor is raked or compressed in which
// round) does not depend on the payload, so one pass carries both the f32
// payload p and an exact uint32 count payload c.
#include <cub/block/block_scan.cuh>
#include <type_traits>
#include "pff_internal.h"

namespace pff {

__global__ void k_rcv2donor_scatter(const int32_t *__restrict__ rcv, int32_t *dnr, int32_t *ndnr, int N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const int r = rcv[t];
    if (r == t) return;
    const int slot = atomicAdd(ndnr + r, 1);
    if (slot < 4) dnr[4 * (long long)r + slot] = t;
}

// Order each node's (at most 4) donor slots by ascending donor index.
__global__ void k_sort_donors(int32_t *dnr, const int32_t *__restrict__ ndnr, int N)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= N) return;
    const int n = min(ndnr[r], 4);
    if (n < 2) return;
    int4 *p4 = reinterpret_cast<int4 *>(dnr) + r;
    int4 v = *p4;
    int d[4] = {v.x, v.y, v.z, v.w};
    for (int a = 1; a < n; ++a) {
        int x = d[a], b = a - 1;
        while (b >= 0 && d[b] > x) { d[b + 1] = d[b]; --b; }
        d[b + 1] = x;
    }
    *p4 = make_int4(d[0], d[1], d[2], d[3]);
}

__device__ __forceinline__ bool get_src(const int32_t *src, int t, int it)
{
    const int e = src[t];
    bool flip = e < 0;
    if (abs(e) == it + 1) flip = !flip;
    return flip;
}

// One rake-and-compress round (downstream_propag.py:157-179).
// If CNT, a second payload c/c_ (uint32) follows the same contraction.
// round_flags (optional): round_flags[it] != 0 if any node worked this round;
// a round whose predecessor did no work returns at once (nothing can change).
template <bool CNT>
__global__ void __launch_bounds__(256) k_rake(int32_t *dnr, int32_t *ndnr, float *p, int32_t *src,
                                              int32_t *dnr_, int32_t *ndnr_, float *p_, uint32_t *c,
                                              uint32_t *c_, int it, int N, int *round_flags)
{
    if (round_flags && it > 0 && *(volatile int *)(round_flags + it - 1) == 0) return;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= N) return;
    const bool flip = get_src(src, tid, it);
    int todo = flip ? ndnr_[tid] : ndnr[tid];
    if (todo <= 0) return;
    const long long base = 4LL * tid;
    const long long lim = 4LL * N;
    int donors[4] = {-1, -1, -1, -1};
    bool worked = false;
    float padd = 0.f;
    uint32_t cadd = 0;
    int i = 0;
    while (i < todo && i < 4) {
        if (donors[i] == -1) donors[i] = flip ? dnr_[base + i] : dnr[base + i];
        const int did = donors[i];
        const bool fd = get_src(src, did, it);
        const int nd = fd ? ndnr_[did] : ndnr[did];
        if (nd <= 1) {
            if (!worked) {
                padd = flip ? p_[tid] : p[tid];
                if (CNT) cadd = flip ? c_[tid] : c[tid];
            }
            worked = true;
            padd = __fadd_rn(padd, fd ? p_[did] : p[did]);
            if (CNT) cadd += fd ? c_[did] : c[did];
            if (nd == 0) {
                --todo;
                if (todo > i && base + todo < lim) donors[i] = flip ? dnr_[base + todo] : dnr[base + todo];
                --i;
            } else {
                donors[i] = fd ? dnr_[4LL * did] : dnr[4LL * did];
            }
        }
        ++i;
    }
    if (!worked) return;
    const int m = todo < 4 ? todo : 4;
    if (flip) {
        ndnr[tid] = todo;
        p[tid] = padd;
        if (CNT) c[tid] = cadd;
        for (int j = 0; j < m; ++j) dnr[base + j] = donors[j];
    } else {
        ndnr_[tid] = todo;
        p_[tid] = padd;
        if (CNT) c_[tid] = cadd;
        for (int j = 0; j < m; ++j) dnr_[base + j] = donors[j];
    }
    src[tid] = (flip ? 1 : -1) * (it + 1);
    if (round_flags) round_flags[it] = 1;
}

template <class T>
__global__ void k_fuse(T *A, const int32_t *__restrict__ src, const T *__restrict__ B, int it, int N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    if (get_src(src, t, it)) A[t] = B[t];
}

__global__ void k_fill_u32(uint32_t *a, uint32_t v, int N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < N) a[t] = v;
}

static int ceil_log2(long long n)
{
    int r = 0;
    long long p = 1;
    while (p < n) { p <<= 1; ++r; }
    return r;
}

// ---------------------------------------------------------------------------
// Whole accumulation with compacted active lists.
//
// The schedule is the reference's rake-and-compress (same rounds, same snapshot
// reads, same per-node donor order), so every f32 sum is formed exactly as in
// the reference; only nodes that still have donors are visited.  Node state:
//   public  {ndnr, p, c, d0}   16 B, read by the node's receiver -> double buffered
//   private {d1, d2, d3, -}    16 B, read and written only by the node itself
// Active nodes rewrite their public record into the next buffer every round;
// a node that finishes in round r has its final record copied into the other
// buffer during round r+1 (that buffer is write-only in round r+1).
struct __align__(16) Pub {
    int ndnr;
    float p;
    uint32_t c;
    int d0;
};

// Fallback path (receivers that are not D4 neighbours): scatter + sort.  Each
// kernel runs only if *need is set (need == nullptr: always).
__global__ void k_acc_init(Pub *A, Pub *B, int4 *priv, const float *__restrict__ Q, uint32_t *counts, int N,
                           const int *need)
{
    if (need && !*need) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        const Pub s{0, Q[t], 1u, -1};
        A[t] = s;
        B[t] = s;
        priv[t] = make_int4(-1, -1, -1, -1);
        if (counts) counts[t] = 1u;
    }
}

__global__ void k_acc_scatter(const int32_t *__restrict__ rcv, Pub *A, int4 *priv, int N, const int *need,
                              int *overflow)
{
    if (need && !*need) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
        const int r = rcv[t];
        if (r == t) continue;
        const int slot = atomicAdd(&A[r].ndnr, 1);
        if (slot == 0) A[r].d0 = t;
        else if (slot < 4) reinterpret_cast<int *>(priv + r)[slot - 1] = t;
        else *overflow = 1;  // more than 4 donors: the reference's slots overflow into the next node's
    }
}

// Block-aggregated append of up to two predicates (order kept within a block).
template <int BS>
__device__ __forceinline__ void block_append2(bool pa, bool pf, int t, int *la, int *na, int *lf, int *nf)
{
    using Scan = cub::BlockScan<int, BS>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int base_a, base_f;
    const int v = (pa ? 1 : 0) | (pf ? 0x10000 : 0);
    int ex, tot;
    Scan(tmp).ExclusiveSum(v, ex, tot);
    if (threadIdx.x == 0) {
        base_a = (tot & 0xFFFF) ? atomicAdd(na, tot & 0xFFFF) : 0;
        base_f = (nf && (tot >> 16)) ? atomicAdd(nf, tot >> 16) : 0;
    }
    __syncthreads();
    if (pa) la[base_a + (ex & 0xFFFF)] = t;
    if (pf) lf[base_f + (ex >> 16)] = t;
    __syncthreads();
}

// Sort each node's donor slots ascending, copy its public record to the second
// buffer, and list the nodes that have donors (round-0 active list).
template <int BS>
__global__ void __launch_bounds__(BS) k_acc_list0(Pub *A, Pub *B, int4 *priv, int *list, int *nlist, int N,
                                                  const int *need)
{
    if (need && !*need) return;
    const int stride = gridDim.x * BS, trips = (N + stride - 1) / stride;
    for (int k = 0; k < trips; ++k) {
    const int t = k * stride + blockIdx.x * BS + threadIdx.x;
    int n = 0;
    if (t < N) {
        Pub s = A[t];
        n = s.ndnr;
        if (n >= 2) {
            int4 q = priv[t];
            int d[4] = {s.d0, q.x, q.y, q.z};
            const int m = n < 4 ? n : 4;
            for (int a = 1; a < m; ++a) {
                int x = d[a], b = a - 1;
                while (b >= 0 && d[b] > x) { d[b + 1] = d[b]; --b; }
                d[b + 1] = x;
            }
            s.d0 = d[0];
            A[t].d0 = d[0];
            priv[t] = make_int4(d[1], d[2], d[3], -1);
        }
        if (n > 0) B[t] = s;
    }
    block_append2<BS>(n > 0, false, t, list, nlist, nullptr, nullptr);
    }
}

// Gather-form initialisation for D4 receivers: the donors of t are the cells
// among its grid neighbours and wrap partners whose receiver is t; visiting
// them in ascending index gives the reference's serial slot order without
// atomics or a sort.  Builds both public buffers, the private slots, the
// counts and the round-0 active list in one pass.  Sets *nonlocal if some
// receiver is not one of these candidates (then the scatter path redoes it).
template <int MODE, int BS>
__global__ void __launch_bounds__(BS) k_acc_gather(const int32_t *__restrict__ rcv, Pub *A, Pub *B, int4 *priv,
                                                   const float *__restrict__ Q, uint32_t *counts, int *list,
                                                   int *nlist, int *nonlocal, int *overflow, Grid g)
{
    const int col = blockIdx.x * 32 + (threadIdx.x & 31);
    const int row = blockIdx.y * (BS / 32) + (threadIdx.x >> 5);
    const bool in = col < g.nx && row < g.ny;
    const int t = row * g.nx + col;
    int nd = 0;
    if (in) {
        const int rt = rcv[t];
        bool ok = rt == t;
        int d[4] = {-1, -1, -1, -1};
        if (MODE != 3) {
            // the neighbour relation of modes 0-2 is symmetric: the donors of t are
            // among its own neighbours; sort them ascending (5 compare-swaps)
            int cn[4];
            neighbours4<MODE>(g, t, row, col, cn);
            int c0 = cn[0], c1 = cn[1], c2 = cn[2], c3 = cn[3];
            // -1 (no neighbour) sorts last
            auto key = [](int v) { return (unsigned)v; };
            auto cs = [&](int &a, int &b) { if (key(a) > key(b)) { int x = a; a = b; b = x; } };
            cs(c0, c1); cs(c2, c3); cs(c0, c2); cs(c1, c3); cs(c1, c2);
            const int cc[4] = {c0, c1, c2, c3};
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const int j = cc[a];
                if (j < 0 || (a > 0 && j == cc[a - 1])) continue;
                if (j == rt) ok = true;
                if (rcv[j] == t) {
                    if (nd < 4) d[nd] = j;
                    ++nd;
                }
            }
        } else {
            int c[8];
            const int n = donor_candidates(g, t, row, col, c);
            for (int a = 0; a < n; ++a) {
                const int j = c[a];
                if (j == rt) ok = true;
                if (rcv[j] == t) {
                    if (nd < 4) d[nd] = j;
                    ++nd;
                }
            }
        }
        if (!ok) *nonlocal = 1;
        if (nd > 4) *overflow = 1;
        const Pub s{nd, Q[t], 1u, d[0]};
        A[t] = s;
        if (nd == 0) {
            // leaves: final from the start, in both buffers; active nodes rewrite B
            // in round 0 and write their counts when they finish
            B[t] = s;
            if (counts) counts[t] = 1u;
        }
        if (nd >= 2) priv[t] = make_int4(d[1], d[2], d[3], -1);
    }
    block_append2<BS>(nd > 0, false, t, list, nlist, nullptr, nullptr);
}

__global__ void k_acc_fallback_reset(int *nlist, const int *need)
{
    if (*need) {
        nlist[0] = 0;  // active and finished counts of round 0
        nlist[1] = 0;
    }
}

__device__ __forceinline__ int sel4(int k, int a, int b, int c, int d)
{
    return k == 0 ? a : (k == 1 ? b : (k == 2 ? c : d));
}
__device__ __forceinline__ void set4(int k, int v, int &a, int &b, int &c, int &d)
{
    a = k == 0 ? v : a;
    b = k == 1 ? v : b;
    c = k == 2 ? v : c;
    d = k == 3 ? v : d;
}
__device__ __forceinline__ Pub pick4(int q, const Pub &a, const Pub &b, const Pub &c, const Pub &d)
{
    return q == 0 ? a : (q == 1 ? b : (q == 2 ? c : d));
}

// One round.  Items [0, nA) are active nodes, [nA, nA+nF) nodes that finished in
// the previous round (copied into the buffer written this round).  In the last
// round (it == logn) every active node reports its start-of-round value, which
// is what the reference's fuse(.., logn) selects (downstream_propag.py:59-74).
// With need != nullptr the round runs only if *need is set (the scatter path's
// rounds before the tile front's first round).  With fin_q, the finished items
// also write their Q and count (the nodes that finished inside the tile front).
template <int BS>
__global__ void __launch_bounds__(BS, 5) k_acc_round(const Pub *__restrict__ cur, Pub *nxt, int4 *priv,
                                                  const int *__restrict__ la, const int *nla,
                                                  const int *__restrict__ lf, const int *nlf, int *la2, int *nla2,
                                                  int *lf2, int *nlf2, float *Q, uint32_t *counts, int it, int last,
                                                  const int *need, int fin_q)
{
    if (need && !*need) return;
    const int nA = *nla, nF = *nlf;
    const int total = nA + nF;
    const int stride = gridDim.x * BS;
    // Uniform trip count so every thread reaches the block-wide appends together.
    // The appends keep each round's list close to ascending order, so the whole
    // GPU works on a narrow window of cells whose donors stay in L2.
    const int trips = (total + stride - 1) / stride;
    for (int k = 0; k < trips; ++k) {
        const int idx = k * stride + blockIdx.x * BS + threadIdx.x;
        bool keep = false, fin = false;
        int t = -1;
        if (idx < nA) {
            t = la[idx];
            const Pub s = cur[t];
            int todo = s.ndnr;
            int own[4] = {s.d0, -1, -1, -1};
            if (todo > 1) {
                const int4 pq = priv[t];
                own[1] = pq.x; own[2] = pq.y; own[3] = pq.z;
            }
            // Every donor state this round can need is one of the start-of-round
            // slots: load them all up front (independent loads).  The reference's
            // swap-remove scan (downstream_propag.py:131-162) then runs on
            // registers: slot k holds donor w_k whose preloaded state is q_k.
            Pub P0 = s, P1 = s, P2 = s, P3 = s;
            if (todo > 0) P0 = cur[own[0]];
            if (todo > 1) P1 = cur[own[1]];
            if (todo > 2) P2 = cur[own[2]];
            if (todo > 3) P3 = cur[own[3]];
            int w0 = own[0], w1 = own[1], w2 = own[2], w3 = own[3];
            int q0 = 0, q1 = 1, q2 = 2, q3 = 3;
            bool worked = false;
            float padd = 0.f;
            uint32_t cadd = 0;
            int i = 0;
#pragma unroll
            for (int step = 0; step < 8; ++step) {  // each step advances i or removes a donor
                if (i >= todo || i >= 4) break;
                const int q = sel4(i, q0, q1, q2, q3);
                const Pub ds = pick4(q, P0, P1, P2, P3);
                if (ds.ndnr <= 1) {
                    if (!worked) { padd = s.p; cadd = s.c; }
                    worked = true;
                    padd = __fadd_rn(padd, ds.p);
                    cadd += ds.c;
                    if (ds.ndnr == 0) {
                        --todo;
                        if (todo > i && todo < 4) {
                            set4(i, sel4(todo, own[0], own[1], own[2], own[3]), w0, w1, w2, w3);
                            set4(i, todo, q0, q1, q2, q3);
                        }
                    } else {
                        set4(i, ds.d0, w0, w1, w2, w3);
                        ++i;
                    }
                } else {
                    ++i;
                }
            }
            const int donors[4] = {w0, w1, w2, w3};
            if (last) {
                Q[t] = s.p;
                if (counts) counts[t] = s.c;
            } else if (!worked) {
                nxt[t] = s;
                keep = true;
            } else {
                nxt[t] = Pub{todo, padd, cadd, todo > 0 ? donors[0] : own[0]};
                if (todo > 1) priv[t] = make_int4(donors[1], donors[2], donors[3], -1);
                if (todo > 0) {
                    keep = true;
                } else {
                    Q[t] = padd;
                    if (counts) counts[t] = cadd;
                    fin = true;
                }
            }
        } else if (idx < total) {
            const int f = lf[idx - nA];
            const Pub s = cur[f];
            nxt[f] = s;
            if (fin_q) {
                Q[f] = s.p;
                if (counts) counts[f] = s.c;
            }
        }
        block_append2<BS>(keep, fin, t, la2, nla2, lf2, nlf2);
    }
}

// ---------------------------------------------------------------------------
// The first FR rounds over spatial tiles (D4 receivers, modes 0-2).
//
// Every donor link joins grid neighbours, and a compress replaces a donor by the
// donor's own donor, so at the start of round r a node's slots point at most 2^r
// hops upstream and its state depends only on the initial states within 2^r - 1
// hops.  The initial state of a cell needs the receivers of its neighbours, one
// more cell.  So one CTA loads a tile plus a halo of 2^FR cells (receivers and
// seeds), builds the initial states in shared memory, and runs the rounds with
// k_acc_round's per-node rule: round r only over the cells within
// 2^FR - 2^(r+1) of the tile (what the later rounds of the tile's cells read),
// the last round in registers for the tile's cells alone.
//
// Outputs, for the tile's cells: the round-FR record in `cur_out` (the buffer
// round FR reads); leaves (no donors ever) also in `nxt_out` with their count 1;
// nodes still active go to the round-FR active list; nodes that finished inside
// the front go to the round-FR finished list, whose copy also writes their Q and
// count (Q is read here as the seeds of neighbouring tiles' halos, so it is
// written only after this launch).  Sets *nonlocal if some receiver is neither
// the cell nor a grid neighbour (then the scatter path redoes everything).
template <int FR>
struct Front {
    static constexpr int H = 1 << FR;
    static constexpr int TW = 64, TH = FR == 1 ? 16 : 24;
    static constexpr int RW = TW + 2 * H, RH = TH + 2 * H, NR = RW * RH;
    static constexpr int BS = 512;
    static constexpr size_t SMEM = (size_t)NR * (6 * 4 + 3 * 2 + 1);
    static_assert(NR < 0xFFFF, "local ids are 16-bit");
    static_assert((TW * TH) % BS == 0, "uniform output trips");
};

// One node's round on shared-memory snapshots (k_acc_round's rule; local ids).
struct FrontNode {
    int todo;
    float p;
    uint32_t c;
    int w0, w1, w2, w3;
    bool worked;
};

__device__ __forceinline__ FrontNode front_round(const float *pc, const uint32_t *cc, const uint32_t *nc,
                                                 uint32_t snd, float sp, uint32_t sc, int own0, int own1, int own2,
                                                 int own3)
{
    constexpr uint32_t NONE = 0xFFFFu;
    int todo = (int)(snd >> 16);
    if (todo == 1) {  // the common chain node: one donor, one step of the rule below
        const uint32_t dn = nc[own0];
        const int dnd = (int)(dn >> 16);
        if (dnd > 1) return FrontNode{1, sp, sc, own0, own1, own2, own3, false};
        const float p = __fadd_rn(sp, pc[own0]);
        const uint32_t c = sc + cc[own0];
        return FrontNode{dnd == 0 ? 0 : 1, p, c, dnd == 0 ? own0 : (int)(dn & NONE), own1, own2, own3, true};
    }
    uint32_t N0 = nc[own0], N1 = snd, N2 = snd, N3 = snd;
    float P0 = pc[own0], P1 = sp, P2 = sp, P3 = sp;
    uint32_t C0 = cc[own0], C1 = sc, C2 = sc, C3 = sc;
    if (todo > 1) { N1 = nc[own1]; P1 = pc[own1]; C1 = cc[own1]; }
    if (todo > 2) { N2 = nc[own2]; P2 = pc[own2]; C2 = cc[own2]; }
    if (todo > 3) { N3 = nc[own3]; P3 = pc[own3]; C3 = cc[own3]; }
    int w0 = own0, w1 = own1, w2 = own2, w3 = own3;
    int q0 = 0, q1 = 1, q2 = 2, q3 = 3;
    bool worked = false;
    float padd = 0.f;
    uint32_t cadd = 0;
    int i = 0;
#pragma unroll
    for (int step = 0; step < 4; ++step) {  // each step moves i up or todo down: todo0 <= 4 steps
        if (i >= todo || i >= 4) break;
        const int q = sel4(i, q0, q1, q2, q3);
        const uint32_t dn = q == 0 ? N0 : (q == 1 ? N1 : (q == 2 ? N2 : N3));
        const float dp = q == 0 ? P0 : (q == 1 ? P1 : (q == 2 ? P2 : P3));
        const uint32_t dc = q == 0 ? C0 : (q == 1 ? C1 : (q == 2 ? C2 : C3));
        const int dnd = (int)(dn >> 16);
        if (dnd <= 1) {
            if (!worked) { padd = sp; cadd = sc; }
            worked = true;
            padd = __fadd_rn(padd, dp);
            cadd += dc;
            if (dnd == 0) {
                --todo;
                if (todo > i && todo < 4) {
                    set4(i, sel4(todo, own0, own1, own2, own3), w0, w1, w2, w3);
                    set4(i, todo, q0, q1, q2, q3);
                }
            } else {
                set4(i, (int)(dn & NONE), w0, w1, w2, w3);
                ++i;
            }
        } else {
            ++i;
        }
    }
    return FrontNode{todo, padd, cadd, w0, w1, w2, w3, worked};
}

template <int MODE, int FR>
__global__ void __launch_bounds__(Front<FR>::BS) k_acc_front(const int32_t *__restrict__ rcv,
                                                              const float *__restrict__ seed, Pub *cur_out,
                                                              Pub *nxt_out, int4 *priv, uint32_t *counts, int *la,
                                                              int *nla, int *lf, int *nlf, int *nonlocal, Grid g,
                                                              int ntx)
{
    using F = Front<FR>;
    constexpr int H = F::H, RW = F::RW, RH = F::RH, NR = F::NR, BS = F::BS, TW = F::TW, TH = F::TH;
    constexpr uint32_t NONE = 0xFFFFu;
    extern __shared__ __align__(16) unsigned char front_sm[];
    __shared__ int rowg[RH], colg[RW];  // global row / column of each region row / column, or -1
    float *pA = reinterpret_cast<float *>(front_sm), *pB = pA + NR;
    uint32_t *cA = reinterpret_cast<uint32_t *>(pB + NR), *cB = cA + NR;
    uint32_t *nA = cB + NR, *nB = nA + NR;  // ndnr << 16 | d0 (local id)
    uint16_t *s1 = reinterpret_cast<uint16_t *>(nB + NR), *s2 = s1 + NR, *s3 = s2 + NR;
    uint8_t *dir = reinterpret_cast<uint8_t *>(s3 + NR);
    const int tx = blockIdx.x % ntx, ty = blockIdx.x / ntx;
    const int c0 = tx * TW - H, r0 = ty * TH - H;  // region origin, before any wrap

    for (int k = threadIdx.x; k < RH + RW; k += BS) {
        if (k < RH) {
            int row = r0 + k;
            if (MODE == 2) {
                row %= g.ny;
                if (row < 0) row += g.ny;
            }
            rowg[k] = (row >= 0 && row < g.ny) ? row : -1;
        } else {
            int col = c0 + k - RH;
            if (MODE == 1) {
                col %= g.nx;
                if (col < 0) col += g.nx;
            }
            colg[k - RH] = (col >= 0 && col < g.nx) ? col : -1;
        }
    }
    __syncthreads();
    auto gid = [&](int lr, int lc) -> int {  // lr, lc within the region
        const int r = rowg[lr], c = colg[lc];
        return (r < 0 || c < 0) ? -1 : r * g.nx + c;
    };
    // a neighbour one step outside the region is never a receiver that matters;
    // -2 keeps it from matching any cell
    auto gidn = [&](int lr, int lc) -> int {
        return (lr < 0 || lr >= RH || lc < 0 || lc >= RW) ? -2 : gid(lr, lc);
    };

    // 1. each cell's receiver as a direction: 0-3 neighbour k, 4 itself, 5 other.
    //    A cell on the region's rim may see its receiver as "other"; it lies
    //    beyond every cell whose state the tile needs.
    bool bad = false;
    for (int x = threadIdx.x; x < NR; x += BS) {
        const int lr = x / RW, lc = x - lr * RW;
        const int t = gid(lr, lc);
        uint8_t d = 5;
        float p = 0.f;
        if (t >= 0) {
            const int rt = rcv[t];
            p = seed[t];
            const int row = rowg[lr], col = colg[lc], dt = rt - t;
            if (rt == t) d = 4;
            else if (row > 0 && row < g.ny - 1 && col > 0 && col < g.nx - 1)  // no wrap or edge next to it
                d = dt == -g.nx ? 0 : (dt == -1 ? 1 : (dt == 1 ? 2 : (dt == g.nx ? 3 : 5)));
            else if (rt == gidn(lr - 1, lc)) d = 0;
            else if (rt == gidn(lr, lc - 1)) d = 1;
            else if (rt == gidn(lr, lc + 1)) d = 2;
            else if (rt == gidn(lr + 1, lc)) d = 3;
            const bool own = lr >= H && lr < H + TH && lc >= H && lc < H + TW && r0 + lr < g.ny && c0 + lc < g.nx;
            if (own && d == 5) bad = true;
        }
        dir[x] = d;
        pA[x] = p;
    }
    if (bad) *nonlocal = 1;
    __syncthreads();

    // 2. initial records within 2^FR - 1 of the tile: the donors are the
    //    neighbours whose receiver is this cell, in ascending global index (wrap
    //    partners can come out of order)
    {
        constexpr int D = H - 1, W = TW + 2 * D, HH = TH + 2 * D;
        for (int u = threadIdx.x; u < W * HH; u += BS) {
            const int lr = u / W + (H - D), lc = u % W + (H - D);
            const int x = lr * RW + lc;
            const int row = rowg[lr], col = colg[lc];
            const bool cell = row >= 0 && col >= 0;
            // candidates in local order top, left, right, bottom: the ascending
            // global order unless a wrap sits next to the cell
            int l0 = NONE, l1 = NONE, l2 = NONE, l3 = NONE;
            if (cell) {
                if (dir[x - RW] == 3) l0 = x - RW;
                if (dir[x - 1] == 2) l1 = x - 1;
                if (dir[x + 1] == 1) l2 = x + 1;
                if (dir[x + RW] == 0) l3 = x + RW;
            }
            const int nd = (l0 != (int)NONE) + (l1 != (int)NONE) + (l2 != (int)NONE) + (l3 != (int)NONE);
            if (nd > 1 && ((MODE == 1 && (col == 0 || col == g.nx - 1)) || (MODE == 2 && (row == 0 || row == g.ny - 1)))) {
                auto key = [&](int l) { return l == (int)NONE ? 0x7FFFFFFF : gid(l / RW, l % RW); };
                int k0 = key(l0), k1 = key(l1), k2 = key(l2), k3 = key(l3);
                auto cs = [](int &ka, int &la_, int &kb, int &lb) {
                    if (ka > kb) {
                        int v = ka; ka = kb; kb = v;
                        v = la_; la_ = lb; lb = v;
                    }
                };
                cs(k0, l0, k1, l1); cs(k2, l2, k3, l3); cs(k0, l0, k2, l2); cs(k1, l1, k3, l3); cs(k1, l1, k2, l2);
            } else {
                // drop the gaps, keeping the order
                if (l0 == (int)NONE) { l0 = l1; l1 = l2; l2 = l3; l3 = NONE; }
                if (l0 == (int)NONE) { l0 = l1; l1 = l2; l2 = NONE; }
                if (l0 == (int)NONE) { l0 = l1; l1 = NONE; }
                if (l1 == (int)NONE) { l1 = l2; l2 = l3; l3 = NONE; }
                if (l1 == (int)NONE) { l1 = l2; l2 = NONE; }
                if (l2 == (int)NONE) { l2 = l3; l3 = NONE; }
            }
            nA[x] = ((uint32_t)nd << 16) | (uint32_t)l0;
            cA[x] = cell ? 1u : 0u;
            s1[x] = (uint16_t)l1;
            s2[x] = (uint16_t)l2;
            s3[x] = (uint16_t)l3;
        }
    }
    __syncthreads();

    // 3. rounds 0..FR-2 within 2^FR - 2^(r+1) of the tile
    float *pc = pA, *pn = pB;
    uint32_t *cc = cA, *cn = cB, *nc = nA, *nn = nB;
#pragma unroll
    for (int r = 0; r < FR - 1; ++r) {
        const int D = H - (2 << r), W = TW + 2 * D, HH = TH + 2 * D;
        for (int u = threadIdx.x; u < W * HH; u += BS) {
            const int x = (u / W + (H - D)) * RW + u % W + (H - D);
            const uint32_t snd = nc[x];
            const float sp = pc[x];
            const uint32_t sc = cc[x];
            if ((snd >> 16) == 0) {
                pn[x] = sp; cn[x] = sc; nn[x] = snd;
                continue;
            }
            const FrontNode o = front_round(pc, cc, nc, snd, sp, sc, (int)(snd & NONE), s1[x], s2[x], s3[x]);
            if (!o.worked) {
                pn[x] = sp; cn[x] = sc; nn[x] = snd;
            } else {
                pn[x] = o.p;
                cn[x] = o.c;
                nn[x] = ((uint32_t)o.todo << 16) | (uint32_t)(o.todo > 0 ? o.w0 : (int)(snd & NONE));
                if (o.todo > 1) {
                    s1[x] = (uint16_t)o.w1;
                    s2[x] = (uint16_t)o.w2;
                    s3[x] = (uint16_t)o.w3;
                }
            }
        }
        __syncthreads();
        float *tp = pc; pc = pn; pn = tp;
        uint32_t *tc = cc; cc = cn; cn = tc;
        uint32_t *tn = nc; nc = nn; nn = tn;
    }

    // 4. round FR-1 for the tile's cells, in registers, then the outputs
    auto l2g = [&](int l) -> int {
        if (l == (int)NONE) return -1;
        const int lr = l / RW;
        return gid(lr, l - lr * RW);
    };
#pragma unroll 1
    for (int k = 0; k < TW * TH / BS; ++k) {
        const int u = k * BS + threadIdx.x;
        const int ir = u / TW, ic = u - ir * TW;
        const int row = ty * TH + ir, col = tx * TW + ic;
        bool act = false, fin = false;
        int t = -1;
        if (row < g.ny && col < g.nx) {
            t = row * g.nx + col;
            const int x = (ir + H) * RW + ic + H;
            const uint32_t snd = nc[x];
            int nd = (int)(snd >> 16);
            float p = pc[x];
            uint32_t c = cc[x];
            int d0 = (int)(snd & NONE), d1 = s1[x], d2 = s2[x], d3 = s3[x];
            if (nd > 0) {
                const FrontNode o = front_round(pc, cc, nc, snd, p, c, d0, d1, d2, d3);
                if (o.worked) {
                    nd = o.todo;
                    p = o.p;
                    c = o.c;
                    if (nd > 0) d0 = o.w0;
                    d1 = o.w1; d2 = o.w2; d3 = o.w3;
                }
            }
            const Pub rec{nd, p, c, nd > 0 ? l2g(d0) : -1};
            cur_out[t] = rec;
            if (nd > 1) priv[t] = make_int4(l2g(d1), nd > 2 ? l2g(d2) : -1, nd > 3 ? l2g(d3) : -1, -1);
            if (nd > 0) {
                act = true;
            } else if (c == 1u) {  // a leaf: it never absorbed a donor
                nxt_out[t] = rec;
                if (counts) counts[t] = 1u;
            } else {
                fin = true;
            }
        }
        block_append2<BS>(act, fin, t, la, nla, lf, nlf);
    }
}

__global__ void k_acc_cond_reset(int *c, const int *need)
{
    if (*need && threadIdx.x < 2) c[threadIdx.x] = 0;
}

template <int MODE, int FR>
static int l_acc_front(const int32_t *rcv, const float *seed, Pub *cur_out, Pub *nxt_out, int4 *priv,
                       uint32_t *counts, int *la, int *nla, int *lf, int *nlf, int *nonlocal, const Grid &g,
                       cudaStream_t st)
{
    using F = Front<FR>;
    static bool attr = false;
    if (!attr) {
        PFF_CUDA(cudaFuncSetAttribute(k_acc_front<MODE, FR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)F::SMEM));
        attr = true;
    }
    const int ntx = div_up(g.nx, F::TW), nty = div_up(g.ny, F::TH);
    { k_acc_front<MODE, FR><<<ntx * nty, F::BS, F::SMEM, st>>>(rcv, seed, cur_out, nxt_out, priv, counts, la, nla, lf,
                                                              nlf, nonlocal, g, ntx); count_launch(); }
    return PFF_OK;
}

// Rounds taken by the tile front (0: off).  A tuning switch; both settings give
// identical results.
static int g_front_rounds = 3;

template <int FR>
static int front_dispatch(int mode, const int32_t *rcv, const float *seed, Pub *cur_out, Pub *nxt_out, int4 *priv,
                          uint32_t *counts, int *la, int *nla, int *lf, int *nlf, int *nonlocal, const Grid &g,
                          cudaStream_t st)
{
    switch (mode) {
    case 0: return l_acc_front<0, FR>(rcv, seed, cur_out, nxt_out, priv, counts, la, nla, lf, nlf, nonlocal, g, st);
    case 1: return l_acc_front<1, FR>(rcv, seed, cur_out, nxt_out, priv, counts, la, nla, lf, nlf, nonlocal, g, st);
    default: return l_acc_front<2, FR>(rcv, seed, cur_out, nxt_out, priv, counts, la, nla, lf, nlf, nonlocal, g, st);
    }
}

__global__ void k_acc_reset_counts(int *c, int n)
{
    if (threadIdx.x < n) c[threadIdx.x] = 0;
}
__global__ void k_acc_fill_one(int *c) { *c = 1; }

template <int MODE>
static void l_acc_gather(const int32_t *rcv, Pub *A, Pub *B, int4 *priv, const float *Q, uint32_t *counts, int *list,
                         int *nlist, int *nonlocal, int *overflow, const Grid &g, cudaStream_t st)
{
    dim3 gr(div_up(g.nx, 32), div_up(g.ny, 8));
    { k_acc_gather<MODE, 256><<<gr, 256, 0, st>>>(rcv, A, B, priv, Q, counts, list, nlist, nonlocal, overflow, g); count_launch(); }
}

}  // namespace pff

using namespace pff;

extern "C" int pff_rcv2donor(const int32_t *rcv, int32_t *dnr, int32_t *ndnr, int N, void *stream)

{
    clear_error();
    if (N <= 0 || !rcv || !dnr || !ndnr || 4LL * N >= (1LL << 31)) {
        set_error("pff_rcv2donor: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_rcv2donor_scatter<<<div_up(N, 256), 256, 0, S(stream)>>>(rcv, dnr, ndnr, N); count_launch(); }
    { k_sort_donors<<<div_up(N, 256), 256, 0, S(stream)>>>(dnr, ndnr, N); count_launch(); }
    return check_cuda("pff_rcv2donor");
}

extern "C" int pff_rake_compress_accum(int32_t *dnr, int32_t *ndnr, float *p, int32_t *src, int32_t *dnr_,
                                       int32_t *ndnr_, float *p_, int iteration, int N, void *stream)
{
    clear_error();
    if (N <= 0 || !dnr || !ndnr || !p || !src || !dnr_ || !ndnr_ || !p_) {
        set_error("pff_rake_compress_accum: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_rake<false><<<div_up(N, 256), 256, 0, S(stream)>>>(dnr, ndnr, p, src, dnr_, ndnr_, p_, nullptr,
                                                        nullptr, iteration, N, nullptr); count_launch(); }
    return check_cuda("pff_rake_compress_accum");
}

extern "C" int pff_fuse(float *A, const int32_t *src, const float *B, int iteration, int N, void *stream)
{
    clear_error();
    if (N <= 0 || !A || !src || !B) {
        set_error("pff_fuse: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_fuse<float><<<div_up(N, 256), 256, 0, S(stream)>>>(A, src, B, iteration, N); count_launch(); }
    return check_cuda("pff_fuse");
}

extern "C" int pff_accumulate_set_front(int rounds)
{
    clear_error();
    if (rounds < 0 || rounds > 3) {
        set_error("pff_accumulate_set_front: rounds must be 0 (off) to 3");
        return PFF_ERR_ARG;
    }
    g_front_rounds = rounds;
    return PFF_OK;
}

extern "C" size_t pff_accumulate_workspace_bytes(int N)
{
    const size_t n = (size_t)N;
    return Carver::round(16 * n) * 3 + Carver::round(4 * n) * 4 + Carver::round(64 * sizeof(int)) + 4096;
}

extern "C" int pff_accumulate(const int32_t *receivers, float *Q, uint32_t *counts, int N, void *workspace,
                              size_t workspace_bytes, void *stream)
{
    return pff_accumulate_grid(receivers, Q, counts, 0, 0, 0, nullptr, N, workspace, workspace_bytes, stream);
}

extern "C" int pff_accumulate_grid(const int32_t *receivers, float *Q, uint32_t *counts, int nx, int ny, int mode,
                                   const uint8_t *codes, int N, void *workspace, size_t workspace_bytes, void *stream)
{
    clear_error();
    if (nx > 0) {
        PFF_TRY(check_grid(nx, ny, mode, codes));
        if (nx * ny != N) {
            set_error("pff_accumulate_grid: N != nx*ny");
            return PFF_ERR_ARG;
        }
    }
    if (N <= 0 || !receivers || !Q || 4LL * N >= (1LL << 31)) {
        set_error("pff_accumulate: bad arguments");
        return PFF_ERR_ARG;
    }
    if (workspace_bytes < pff_accumulate_workspace_bytes(N) || !workspace) {
        set_error("pff_accumulate: workspace too small (%zu < %zu)", workspace_bytes,
                  pff_accumulate_workspace_bytes(N));
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    Carver cv(workspace, workspace_bytes);
    Pub *A = cv.take<Pub>(N);
    Pub *B = cv.take<Pub>(N);
    int4 *priv = cv.take<int4>(N);
    int *lA0 = cv.take<int>(N), *lA1 = cv.take<int>(N), *lF0 = cv.take<int>(N), *lF1 = cv.take<int>(N);
    int *ctr = cv.take<int>(64);  // [2*r] active count, [2*r+1] finished count, by round parity
    constexpr int BS = 256;
    const int logn = ceil_log2(N) + 1;  // flowfields.py:272
    const int FR = g_front_rounds;
    const bool front = nx > 0 && mode >= 0 && mode <= 2 && nx >= 3 && ny >= 3 && FR > 0 && logn > FR;
    { k_acc_reset_counts<<<1, 64, 0, st>>>(ctr, 64); count_launch(); }
    int *nonlocal = ctr + 63, *overflow = ctr + 62;
    Pub *bufs[2] = {A, B};
    int *la[2] = {lA0, lA1}, *lf[2] = {lF0, lF1};
    if (front) {
        Grid g{nx, ny, mode, codes};
        const int pa = FR & 1;
        int *na = ctr + 4 * pa;
        auto run = [&](auto fr) {
            return front_dispatch<decltype(fr)::value>(mode, receivers, Q, bufs[pa], bufs[pa ^ 1], priv, counts,
                                                       la[pa], na, lf[pa], na + 1, nonlocal, g, st);
        };
        PFF_TRY(FR == 1 ? run(std::integral_constant<int, 1>{})
                        : (FR == 2 ? run(std::integral_constant<int, 2>{}) : run(std::integral_constant<int, 3>{})));
    } else if (nx > 0) {
        Grid g{nx, ny, mode, codes};
        PFF_MODE_DISPATCH(mode, l_acc_gather, receivers, A, B, priv, Q, counts, lA0, ctr + 0, nonlocal, overflow, g,
                          st);
    } else {
        { k_acc_fill_one<<<1, 1, 0, st>>>(nonlocal); count_launch(); }
    }
    // receivers that are not D4 neighbours (or no grid given): scatter path
    { k_acc_fallback_reset<<<1, 1, 0, st>>>(ctr + 0, nonlocal); count_launch(); }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * 8;
    { k_acc_init<<<grid, BS, 0, st>>>(A, B, priv, Q, counts, N, nonlocal); count_launch(); }
    { k_acc_scatter<<<grid, BS, 0, st>>>(receivers, A, priv, N, nonlocal, overflow); count_launch(); }
    { k_acc_list0<BS><<<grid, BS, 0, st>>>(A, B, priv, lA0, ctr + 0, N, nonlocal); count_launch(); }
    static int round_blocks = 0;
    if (!round_blocks) {
        int per = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_acc_round<BS>, BS, 0);
        round_blocks = nsm * (per > 0 ? per : 1);
    }
    for (int it = 0; it <= logn; ++it) {
        const int a = it & 1, b = a ^ 1;
        // list counters: ctr[4*parity] = active, ctr[4*parity+1] = finished
        int *na_in = ctr + 4 * a, *nf_in = na_in + 1;
        int *na_out = ctr + 4 * b, *nf_out = na_out + 1;
        // with the tile front, rounds 0..FR-1 run only on the scatter path
        const bool cond = front && it < FR;
        if (cond) {
            { k_acc_cond_reset<<<1, 32, 0, st>>>(na_out, nonlocal); count_launch(); }
        } else {
            PFF_CUDA(cudaMemsetAsync(na_out, 0, 2 * sizeof(int), st));
        }
        { k_acc_round<BS><<<round_blocks, BS, 0, st>>>(bufs[a], bufs[b], priv, la[a], na_in, lf[a], nf_in, la[b], na_out,
                                               lf[b], nf_out, Q, counts, it, it == logn, cond ? nonlocal : nullptr,
                                               front && it == FR); count_launch(); }
    }
    PFF_TRY(check_cuda("pff_accumulate"));
    int over = 0;
    PFF_TRY(read_ints(IntReads().add(overflow, 1), &over, st));
    if (over) {
        set_error("pff_accumulate: a node has more than 4 donors (possible only after jump rerouting); "
                  "the reference's donor slots overflow there and this case is not supported");
        return PFF_ERR_ARG;
    }
    return PFF_OK;
}
