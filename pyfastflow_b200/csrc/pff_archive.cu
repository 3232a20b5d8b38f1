// libpff legacy downstream tree algorithms of pyfastflow's archive (the CUDA
// kernels the package was first written around, archive/fastflow/kernels):
//   tree_accum_down  x_i = p_i + W_i * x_rcv(i), solved by pointer jumping
//   tree_max_down    the largest value on each cell's downstream path
//   erode_deposit    deposition + implicit stream-power erosion, whose elevation
//                    update is a tree_accum_down solve
// Each round reads the start-of-round arrays (the reference double-buffers them
// and copies back after every round), so the f32 results are the reference's
// operation for operation.  The jumping runs ceil(log2 N) rounds like the
// reference's drivers; rcv, W and p are left as those drivers leave them.
#include "pff_internal.h"

namespace pff {

// tree_accum_down.py:15-21
__global__ void k_tad_round(const int32_t *__restrict__ rcv, const float *__restrict__ W,
                            const float *__restrict__ p, int32_t *__restrict__ r2, float *__restrict__ W2,
                            float *__restrict__ p2, int N, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int r = rcv[i];
    if (r < 0 || r >= N) { atomicOr(err, 1); r = i; }
    const float wi = W[i];
    p2[i] = __fadd_rn(p[i], __fmul_rn(wi, p[r]));
    W2[i] = __fmul_rn(wi, W[r]);
    const int rr = rcv[r];
    r2[i] = (rr < 0 || rr >= N) ? r : rr;
}

// tree_max_down.py:7-12; max(a, b) = a > b ? a : b
__global__ void k_tmd_round(const int32_t *__restrict__ rcv, const float *__restrict__ p, int32_t *__restrict__ r2,
                            float *__restrict__ p2, int N, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int r = rcv[i];
    if (r < 0 || r >= N) { atomicOr(err, 1); r = i; }
    const int rr = rcv[r];
    if (rr >= 0 && rr < N && rr != r) {
        const float a = p[r], b = p[i];
        p2[i] = a > b ? a : b;
        r2[i] = rr;
    } else {
        p2[i] = p[i];
        r2[i] = r;
    }
}

// erode_deposit.py:7-24; powers in double, rounded once to f32
__global__ void k_erode_deposit(float *z, const uint8_t *__restrict__ bound, const float *__restrict__ drain,
                                const float *__restrict__ Qs, float dt, float dx, float k_spl, float k_t, float k_h,
                                float k_d, float m, float *pe, float *We, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    float zi = z[i];
    const float d = drain[i];
    const bool b = bound[i] != 0;
    if (!b) {
        const float cd = fminf(__fdiv_rn(k_d, d), 1.0f);
        zi = __fadd_rn(zi, __fmul_rn(__fmul_rn(dt, cd), Qs[i]));
        z[i] = zi;
    }
    const float pm = (float)pow((double)d, (double)m);
    const float pmm = (float)pow((double)d, (double)(-m));
    float s = __fmul_rn(k_spl, pm);
    s = __fadd_rn(s, k_t);
    s = __fadd_rn(s, __fmul_rn(k_h, pmm));
    const float K = __fmul_rn(__fdiv_rn(dt, dx), s);
    const float one_k = __fadd_rn(1.0f, K);
    pe[i] = b ? zi : __fdiv_rn(zi, one_k);
    We[i] = b ? 0.0f : __fdiv_rn(K, one_k);
}

static int rounds_for(int N)
{
    int r = 0;
    long long q = 1;
    while (q < N) { q <<= 1; ++r; }
    return r;
}

struct ArchWs {
    int32_t *r2;
    float *a2, *b2;
    int *err;
};
static ArchWs arch_ws(void *ws, size_t bytes, int N)
{
    Carver cv(ws, bytes);
    ArchWs w;
    w.r2 = cv.take<int32_t>(N);
    w.a2 = cv.take<float>(N);
    w.b2 = cv.take<float>(N);
    w.err = cv.take<int>(64);
    return w;
}

// rounds of tree_accum_down on (rcv, W, p) in place, ping-ponging with the workspace
static int tad_rounds(int32_t *rcv, float *W, float *p, int N, const ArchWs &w, cudaStream_t st)
{
    const int R = rounds_for(N);
    int32_t *ra = rcv, *rb = w.r2;
    float *Wa = W, *Wb = w.a2, *pa = p, *pb = w.b2;
    for (int it = 0; it < R; ++it) {
        { k_tad_round<<<div_up(N, 256), 256, 0, st>>>(ra, Wa, pa, rb, Wb, pb, N, w.err); count_launch(); }
        std::swap(ra, rb);
        std::swap(Wa, Wb);
        std::swap(pa, pb);
    }
    if (ra != rcv) {  // an odd number of rounds: the caller's arrays hold the last results
        PFF_CUDA(cudaMemcpyAsync(rcv, ra, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToDevice, st));
        PFF_CUDA(cudaMemcpyAsync(W, Wa, sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, st));
        PFF_CUDA(cudaMemcpyAsync(p, pa, sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    }
    return check_cuda("tree_accum_down");
}

static int read_err(const ArchWs &w, const char *who, cudaStream_t st)
{
    int e = 0;
    PFF_TRY(read_ints(IntReads().add(w.err, 1), &e, st));
    if (e) {
        set_error("%s: a receiver index is out of range", who);
        return PFF_ERR_ARG;
    }
    return PFF_OK;
}

}  // namespace pff

using namespace pff;

extern "C" size_t pff_archive_workspace_bytes(int N)
{
    if (N < 1) return 0;
    return Carver::round(4 * (size_t)N) * 3 + Carver::round(sizeof(int) * 64) + 1024;
}

extern "C" int pff_tree_accum_down(int32_t *rcv, float *W, float *p, int N, void *workspace, size_t workspace_bytes,
                                   void *stream)
{
    clear_error();
    if (N < 1 || !rcv || !W || !p) {
        set_error("pff_tree_accum_down: bad arguments");
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_archive_workspace_bytes(N)) {
        set_error("pff_tree_accum_down: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    ArchWs w = arch_ws(workspace, workspace_bytes, N);
    PFF_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    PFF_TRY(tad_rounds(rcv, W, p, N, w, st));
    return read_err(w, "pff_tree_accum_down", st);
}

extern "C" int pff_tree_max_down(int32_t *rcv, float *p, int N, void *workspace, size_t workspace_bytes, void *stream)
{
    clear_error();
    if (N < 1 || !rcv || !p) {
        set_error("pff_tree_max_down: bad arguments");
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_archive_workspace_bytes(N)) {
        set_error("pff_tree_max_down: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    ArchWs w = arch_ws(workspace, workspace_bytes, N);
    PFF_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    const int R = rounds_for(N);
    int32_t *ra = rcv, *rb = w.r2;
    float *pa = p, *pb = w.b2;
    for (int it = 0; it < R; ++it) {
        { k_tmd_round<<<div_up(N, 256), 256, 0, st>>>(ra, pa, rb, pb, N, w.err); count_launch(); }
        std::swap(ra, rb);
        std::swap(pa, pb);
    }
    if (ra != rcv) {
        PFF_CUDA(cudaMemcpyAsync(rcv, ra, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToDevice, st));
        PFF_CUDA(cudaMemcpyAsync(p, pa, sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, st));
    }
    PFF_TRY(check_cuda("pff_tree_max_down"));
    return read_err(w, "pff_tree_max_down", st);
}

extern "C" int pff_erode_deposit(float *z, const uint8_t *bound, int32_t *rcv, const float *drain, const float *Qs,
                                 float dt, float dx, float k_spl, float k_t, float k_h, float k_d, float m, float *pe,
                                 float *We, int N, void *workspace, size_t workspace_bytes, void *stream)
{
    clear_error();
    if (N < 1 || !z || !bound || !rcv || !drain || !Qs || !pe || !We) {
        set_error("pff_erode_deposit: bad arguments");
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_archive_workspace_bytes(N)) {
        set_error("pff_erode_deposit: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    ArchWs w = arch_ws(workspace, workspace_bytes, N);
    PFF_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    { k_erode_deposit<<<div_up(N, 256), 256, 0, st>>>(z, bound, drain, Qs, dt, dx, k_spl, k_t, k_h, k_d, m, pe, We,
                                                      N); count_launch(); }
    PFF_TRY(tad_rounds(rcv, We, pe, N, w, st));
    return read_err(w, "pff_erode_deposit", st);
}
