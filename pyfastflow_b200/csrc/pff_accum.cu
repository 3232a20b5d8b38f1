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
    size_t n = (size_t)N;
    return Carver::round(16 * n) * 2 + Carver::round(4 * n) * 5 + Carver::round(64 * 4) + 4096;
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
    int32_t *dnr = cv.take<int32_t>(4 * (size_t)N);
    int32_t *dnr_ = cv.take<int32_t>(4 * (size_t)N);
    int32_t *ndnr = cv.take<int32_t>(N);
    int32_t *ndnr_ = cv.take<int32_t>(N);
    int32_t *src = cv.take<int32_t>(N);
    float *Q_ = cv.take<float>(N);
    uint32_t *c_ = cv.take<uint32_t>(N);
    int *flags = cv.take<int>(64);
    const int logn = ceil_log2(N) + 1;  // flowfields.py:272
    PFF_CUDA(cudaMemsetAsync(ndnr, 0, sizeof(int32_t) * (size_t)N, st));
    PFF_CUDA(cudaMemsetAsync(src, 0, sizeof(int32_t) * (size_t)N, st));
    PFF_CUDA(cudaMemsetAsync(flags, 0, sizeof(int) * 64, st));
    const int nb = div_up(N, 256);
    if (counts) { k_fill_u32<<<nb, 256, 0, st>>>(counts, 1u, N); count_launch(); }
    { k_rcv2donor_scatter<<<nb, 256, 0, st>>>(receivers, dnr, ndnr, N); count_launch(); }
    { k_sort_donors<<<nb, 256, 0, st>>>(dnr, ndnr, N); count_launch(); }
    for (int it = 0; it <= logn; ++it) {
        if (counts)
            { k_rake<true><<<nb, 256, 0, st>>>(dnr, ndnr, Q, src, dnr_, ndnr_, Q_, counts, c_, it, N, flags); count_launch(); }
        else
            { k_rake<false><<<nb, 256, 0, st>>>(dnr, ndnr, Q, src, dnr_, ndnr_, Q_, nullptr, nullptr, it, N, flags); count_launch(); }
    }
    { k_fuse<float><<<nb, 256, 0, st>>>(Q, src, Q_, logn, N); count_launch(); }
    if (counts) { k_fuse<uint32_t><<<nb, 256, 0, st>>>(counts, src, c_, logn, N); count_launch(); }
    return check_cuda("pff_accumulate");
}
