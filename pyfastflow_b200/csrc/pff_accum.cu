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

__global__ void k_acc_init(Pub *A, Pub *B, int4 *priv, const float *__restrict__ Q, uint32_t *counts, int N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const Pub s{0, Q[t], 1u, -1};
    A[t] = s;
    B[t] = s;
    priv[t] = make_int4(-1, -1, -1, -1);
    if (counts) counts[t] = 1u;
}

__global__ void k_acc_scatter(const int32_t *__restrict__ rcv, Pub *A, int4 *priv, int N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    const int r = rcv[t];
    if (r == t) return;
    const int slot = atomicAdd(&A[r].ndnr, 1);
    if (slot == 0) A[r].d0 = t;
    else if (slot < 4) reinterpret_cast<int *>(priv + r)[slot - 1] = t;
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
__global__ void __launch_bounds__(BS) k_acc_list0(Pub *A, Pub *B, int4 *priv, int *list, int *nlist, int N)
{
    const int t = blockIdx.x * BS + threadIdx.x;
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

// One round.  Items [0, nA) are active nodes, [nA, nA+nF) nodes that finished in
// the previous round (copied into the buffer written this round).  In the last
// round (it == logn) every active node reports its start-of-round value, which
// is what the reference's fuse(.., logn) selects (downstream_propag.py:59-74).
template <int BS>
__global__ void __launch_bounds__(BS) k_acc_round(const Pub *__restrict__ cur, Pub *nxt, int4 *priv,
                                                  const int *__restrict__ la, const int *nla,
                                                  const int *__restrict__ lf, const int *nlf, int *la2, int *nla2,
                                                  int *lf2, int *nlf2, float *Q, uint32_t *counts, int it, int last)
{
    const int nA = *nla, nF = *nlf;
    const int total = nA + nF;
    const int stride = gridDim.x * BS;
    // uniform trip count so every thread reaches the block-wide appends together
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
                const int4 q = priv[t];
                own[1] = q.x; own[2] = q.y; own[3] = q.z;
            }
            int donors[4] = {-1, -1, -1, -1};
            bool worked = false;
            float padd = 0.f;
            uint32_t cadd = 0;
            int i = 0;
            while (i < todo && i < 4) {
                if (donors[i] == -1) donors[i] = own[i];
                const int did = donors[i];
                const Pub ds = cur[did];
                if (ds.ndnr <= 1) {
                    if (!worked) { padd = s.p; cadd = s.c; }
                    worked = true;
                    padd = __fadd_rn(padd, ds.p);
                    cadd += ds.c;
                    if (ds.ndnr == 0) {
                        --todo;
                        if (todo > i && todo < 4) donors[i] = own[todo];
                        --i;
                    } else {
                        donors[i] = ds.d0;
                    }
                }
                ++i;
            }
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
            nxt[f] = cur[f];
        }
        block_append2<BS>(keep, fin, t, la2, nla2, lf2, nlf2);
    }
}

__global__ void k_acc_reset_counts(int *c, int n)
{
    if (threadIdx.x < n) c[threadIdx.x] = 0;
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

extern "C" size_t pff_accumulate_workspace_bytes(int N)
{
    const size_t n = (size_t)N;
    return Carver::round(16 * n) * 3 + Carver::round(4 * n) * 4 + Carver::round(64 * sizeof(int)) + 4096;
}

extern "C" int pff_accumulate(const int32_t *receivers, float *Q, uint32_t *counts, int N, void *workspace,
                              size_t workspace_bytes, void *stream)
{
    clear_error();
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
    const int nb = div_up(N, BS);
    const int logn = ceil_log2(N) + 1;  // flowfields.py:272
    { k_acc_reset_counts<<<1, 64, 0, st>>>(ctr, 64); count_launch(); }
    { k_acc_init<<<nb, BS, 0, st>>>(A, B, priv, Q, counts, N); count_launch(); }
    { k_acc_scatter<<<nb, BS, 0, st>>>(receivers, A, priv, N); count_launch(); }
    { k_acc_list0<BS><<<nb, BS, 0, st>>>(A, B, priv, lA0, ctr + 0, N); count_launch(); }
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * 8;
    Pub *bufs[2] = {A, B};
    int *la[2] = {lA0, lA1}, *lf[2] = {lF0, lF1};
    for (int it = 0; it <= logn; ++it) {
        const int a = it & 1, b = a ^ 1;
        // list counters: ctr[4*parity] = active, ctr[4*parity+1] = finished
        int *na_in = ctr + 4 * a, *nf_in = na_in + 1;
        int *na_out = ctr + 4 * b, *nf_out = na_out + 1;
        PFF_CUDA(cudaMemsetAsync(na_out, 0, 2 * sizeof(int), st));
        { k_acc_round<BS><<<grid, BS, 0, st>>>(bufs[a], bufs[b], priv, la[a], na_in, lf[a], nf_in, la[b], na_out,
                                               lf[b], nf_out, Q, counts, it, it == logn); count_launch(); }
    }
    return check_cuda("pff_accumulate");
}
