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
#include "pff_internal.h"

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
__global__ void k_basin_init(int32_t *bid, Grid g)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.N()) return;
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

// ---- launchers ---------------------------------------------------------------

template <int MODE>
static void l_count_pits(const int32_t *rec, const Grid &g, int *count, int *list, cudaStream_t st)
{
    { k_count_pits<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(rec, g, count, list); count_launch(); }
}
template <int MODE>
static void l_basin_init(int32_t *bid, const Grid &g, cudaStream_t st)
{
    { k_basin_init<MODE><<<div_up(g.N(), 256), 256, 0, st>>>(bid, g); count_launch(); }
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
    if (host_count) {
        PFF_CUDA(cudaMemcpyAsync(host_count, dev_count, sizeof(int), cudaMemcpyDeviceToHost, st));
        PFF_CUDA(cudaStreamSynchronize(st));
    }
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
    return Carver::round((size_t)N + 1) + Carver::round(sizeof(int) * (size_t)N) + Carver::round(sizeof(int) * 256) + 4096;
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
    Carver cv(workspace, workspace_bytes);
    uint8_t *inv = cv.take<uint8_t>((size_t)N + 1);
    int *pits = cv.take<int>(N);
    int *ctr = cv.take<int>(256);  // [0] pit count, [64..127] label flags, [128..191] carve flags
    int *lflags = ctr + 64, *cflags = ctr + 128;
    long long *sad = (long long *)basin_saddle, *out = (long long *)outlet;
    const size_t nb4 = sizeof(int32_t) * (size_t)N;
    const int B = 256, nbk = div_up(N, B);
    if (n_outer_out) *n_outer_out = 0;

    PFF_CUDA(cudaMemcpyAsync(rec_, rec, nb4, cudaMemcpyDeviceToDevice, st));  // :491
    int Ndep = 0;
    PFF_TRY(count_pits(rec, g, ctr, nullptr, &Ndep, st));  // :493
    if (Ndep == 0) return PFF_OK;
    const int outer = ceil_log2(Ndep) + 1;  // :500
    const int carve_rounds = ceil_log2(N) + 2;
    int n_outer = 0;
    for (int it = 0; it < outer; ++it) {
        int nd_bis = 0;
        PFF_TRY(count_pits(rec_, g, ctr, nullptr, &nd_bis, st));  // :501
        PFF_TRY(launch_basin_init(bid, g, st));                   // :507
        PFF_CUDA(cudaMemcpyAsync(rec__, rec_, nb4, cudaMemcpyDeviceToDevice, st));
        PFF_TRY(run_labels(bid, rec__, g, lflags, st));  // :510-511
        ++n_outer;
        if (nd_bis == 0) break;  // :512
        PFF_MODE_DISPATCH(bound_mode, l_saddle, bid, is_border, z_prime, sad, basin_saddlenode, out, inv, z, g, st);
        if (carve) {
            // reroute_carve :424-438
            PFF_CUDA(cudaMemsetAsync(tag, 0, (size_t)N, st));
            { k_carve_tag_saddles<<<nbk, B, 0, st>>>(basin_saddlenode, tag, N); count_launch(); }
            PFF_CUDA(cudaMemcpyAsync(tag_, tag, (size_t)N, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemcpyAsync(rec, rec_, nb4, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemcpyAsync(rec__, rec_, nb4, cudaMemcpyDeviceToDevice, st));
            PFF_CUDA(cudaMemsetAsync(cflags, 0, sizeof(int) * 64, st));
            for (int r = 0; r < carve_rounds; ++r) {
                { k_carve_it1<<<nbk, B, 0, st>>>(tag, tag_, rec, rec_, N, r, cflags); count_launch(); }
                { k_carve_it2<<<nbk, B, 0, st>>>(tag, tag_, rec, rec_, N, r, cflags); count_launch(); }
            }
            PFF_CUDA(cudaMemcpyAsync(rec, rec__, nb4, cudaMemcpyDeviceToDevice, st));
            { k_carve_reverse<<<nbk, B, 0, st>>>(rec, rec__, tag, N); count_launch(); }
            { k_carve_link_outlets<<<nbk, B, 0, st>>>(rec, basin_saddlenode, out, N, 0); count_launch(); }
            PFF_CUDA(cudaMemcpyAsync(rec_, rec, nb4, cudaMemcpyDeviceToDevice, st));  // :526
        } else {
            { k_carve_link_outlets<<<nbk, B, 0, st>>>(rec_, basin_saddlenode, out, N, 1); count_launch(); }  // :529
        }
        PFF_TRY(check_cuda("pff_reroute_flow"));
    }
    PFF_TRY(launch_basin_init(bid, g, st));  // :537
    if (n_outer_out) *n_outer_out = n_outer;
    return check_cuda("pff_reroute_flow");
}
