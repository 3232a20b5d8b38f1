// libpff GraphFlood: topographic fill with delta, MFD discharge diffusion and
// the Manning depth update (pyfastflow/flow/fill_topo.py, graphflood/gf_hydrodynamics.py).
//
// All f32 arithmetic is written with explicit round-to-nearest intrinsics (and
// the library is built with -fmad=false), so each operation is the reference's
// single IEEE operation in the reference's order.
#include <algorithm>
#include <cstdlib>
#include "pff_internal.h"
#include "pff_div.cuh"

namespace pff {

// ---- fill (fill_topo.py:17-45, snapshot semantics) ---------------------------
__global__ void __launch_bounds__(256) k_fill_round(const float *__restrict__ zh, const float *__restrict__ zs,
                                                    float *__restrict__ zn, const int32_t *__restrict__ ra,
                                                    int32_t *__restrict__ rb, float inc, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int r = ra[i];
    const int rr = ra[r];
    rb[i] = rr;                                            // :29
    const float zi = zs[i];
    if (i == r || (zi > zh[r] && rr == r)) { zn[i] = zi; return; }  // :32
    zn[i] = fmaxf(zi, __fadd_rn(zs[r], inc));              // :36
}

// The same rounds on one 8-byte record per cell, {pointer, snapshot z}: a round reads
// its own record and gathers the record at its pointer (one sector instead of three
// gathers), then writes its new record.  zh[r] is needed only where r points to
// itself; at a cell whose receiver is itself from the start, the snapshot never
// changes (:32 keeps it), so zs[r] is zh[r] there.  Bit 31 of the pointer word marks
// those cells; a self-pointer made by a receiver cycle (no such bit) reads zh[r].
constexpr uint32_t FILL_ROOT = 0x80000000u;
// Rounds from FILL_VOTE0 on record whether any input record was unsettled; a round
// after one whose input was all settled does nothing (see k_fill_round_packed).
constexpr int FILL_VOTE0 = 10;
constexpr int FILL_FLAGS = 64;  // ints after the two record buffers in the workspace
__global__ void __launch_bounds__(256) k_fill_pack(const float *__restrict__ zh, const int32_t *__restrict__ rcv,
                                                   uint2 *__restrict__ A, int N, int *flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (flags && blockIdx.x == 0 && threadIdx.x < FILL_FLAGS) flags[threadIdx.x] = 0;
    if (i >= N) return;
    int r = rcv[i];
    if ((unsigned)r >= (unsigned)N) r = i;  // an out-of-range receiver: no read outside the records
    A[i] = make_uint2((uint32_t)r | (r == i ? FILL_ROOT : 0u), __float_as_uint(zh[i]));
}

// One round for cell i: `me` its record, `at` the record at its pointer.  `settled`:
// the cell is a root, or its pointer reaches a root (rr == r) and it stands above
// that root's surface, so it keeps its record in this and every later round,
// whatever the increment.
__device__ __forceinline__ uint2 fill_step(const float *__restrict__ zh, int i, uint2 me, uint2 at, float inc,
                                           bool &settled)
{
    const int r = (int)(me.x & ~FILL_ROOT);
    const int rr = (int)(at.x & ~FILL_ROOT);
    const float zi = __uint_as_float(me.y), zr = __uint_as_float(at.y);
    float zn;
    settled = true;
    if (i == r) zn = zi;
    else if (rr == r && zi > ((at.x & FILL_ROOT) ? zr : zh[r])) zn = zi;  // :32
    else {
        zn = fmaxf(zi, __fadd_rn(zr, inc));                               // :36
        settled = false;
    }
    return make_uint2((uint32_t)rr | (me.x & FILL_ROOT), __float_as_uint(zn));  // :29
}

// FILL_CPT cells per thread (i, i + 256, ... in a block's 256 * FILL_CPT): all their
// records are read, then all the gathers at their pointers are in flight at once (the
// rounds are bound by the latency of that dependent gather).  Returns whether any
// input record was unsettled.
constexpr int FILL_CPT = 4;
__device__ __forceinline__ bool fill_cells(const float *__restrict__ zh, const uint2 *__restrict__ A,
                                           uint2 *__restrict__ B, float inc, int N, int base)
{
    uint2 m[FILL_CPT], at[FILL_CPT];
#pragma unroll
    for (int k = 0; k < FILL_CPT; ++k) {
        const int i = base + threadIdx.x + 256 * k;
        m[k] = i < N ? A[i] : make_uint2(0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < FILL_CPT; ++k) {
        const int i = base + threadIdx.x + 256 * k;
        at[k] = i < N ? A[m[k].x & ~FILL_ROOT] : make_uint2(0u, 0u);
    }
    bool uns = false;
#pragma unroll
    for (int k = 0; k < FILL_CPT; ++k) {
        const int i = base + threadIdx.x + 256 * k;
        if (i < N) {
            bool st;
            B[i] = fill_step(zh, i, m[k], at[k], inc, st);
            uns |= !st;
        }
    }
    return uns;
}

__global__ void __launch_bounds__(256) k_fill_round_packed(const float *__restrict__ zh, const uint2 *__restrict__ A,
                                                           uint2 *__restrict__ B, float inc, int N)
{
    fill_cells(zh, A, B, inc, N, blockIdx.x * (256 * FILL_CPT));
}

// The rounds from FILL_VOTE0 on: the same step over a grid-stride loop with a few
// blocks per SM, each block recording in flags[it] whether any input record it read
// was unsettled (one atomic per block at most, after a read of the flag).  If the
// input of round it-1 was all settled, round it-1 copied every record unchanged and
// so would every later round: round it then returns at once (both record buffers
// already hold the final records), as do the later rounds, whose flags stay 0.
__global__ void __launch_bounds__(256) k_fill_round_late(const float *__restrict__ zh, const uint2 *__restrict__ A,
                                                         uint2 *__restrict__ B, float inc, int N, int *flags, int it)
{
    if (it > FILL_VOTE0 && *(volatile const int *)&flags[it - 1] == 0) return;
    bool uns = false;
    for (int base = blockIdx.x * (256 * FILL_CPT); base < N; base += gridDim.x * (256 * FILL_CPT))
        uns |= fill_cells(zh, A, B, inc, N, base);
    if (__syncthreads_or(uns) && threadIdx.x == 0 && *(volatile int *)&flags[it] == 0) atomicOr(&flags[it], 1);
}

// the packed result to z_ and both receiver buffers (:39-40), then, if h is given,
// _apply_fill_z_add_delta (:82-97); write_z copies z_ into zh without a depth update
__global__ void __launch_bounds__(256) k_fill_unpack(const uint2 *__restrict__ A, float *z_, int32_t *r1, int32_t *r2,
                                                     float *zh, float *h, bool write_z, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const uint2 a = A[i];
    const int r = (int)(a.x & ~FILL_ROOT);
    const float zf = __uint_as_float(a.y);
    z_[i] = zf;
    r1[i] = r;
    r2[i] = r;
    if (h) h[i] = __fadd_rn(h[i], __fsub_rn(zf, zh[i]));
    if (h || write_z) zh[i] = zf;
}

// _apply_fill_z_add_delta (:82-97)
__global__ void k_fill_apply(float *zh, float *h, const float *__restrict__ z_, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const float zf = z_[i];
    h[i] = __fadd_rn(h[i], __fsub_rn(zf, zh[i]));
    zh[i] = zf;
}

// ---- diffusion (gf_hydrodynamics.py:24-75) -----------------------------------
// Per-cell outgoing weights fl(tS_k / sums) and a "source" flag (non-outlet
// with sums != 0), computed once per call: zh does not change between sweeps.
template <int MODE>
__global__ void __launch_bounds__(256) k_diffuse_weights(const float *__restrict__ zh, float *w, uint8_t *issrc,
                                                         Grid g, float dx)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= g.nx || row >= g.ny) return;
    const int i = row * g.nx + col;
    if (can_leave<MODE>(g, i, row, col)) { issrc[i] = 0; return; }
    const float zi = zh[i];
    float s[4];
    float sums = 0.f;
    int js[4];
    neighbours4<MODE>(g, i, row, col, js);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = js[k];
        s[k] = (j != -1) ? fmaxf(0.f, __fdiv_rn(__fsub_rn(zi, zh[j]), dx)) : 0.f;
        sums = __fadd_rn(sums, s[k]);  // j == -1 adds max(0, 0) = 0
    }
    if (sums == 0.f) { issrc[i] = 0; return; }
    issrc[i] = 1;
    // one plane per direction k: a gather reads only the weight it needs
    const size_t N = (size_t)g.N();
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k * N + i] = __fdiv_rn(s[k], sums);
}

// One sweep in gather form: temp[j] = P*dx^2 + sum over sources i ascending, then
// k ascending, of fl(w_ik * Q[i]) -- the serial order of the reference's atomics.
// Interior cells of modes 0-2: the sources are the top, left, right and bottom
// neighbours (ascending index), each reaching j through its bottom, right, left
// and top link respectively.
template <int MODE>
__global__ void __launch_bounds__(256) k_diffuse_sweep(const float *__restrict__ Q, float *__restrict__ Qn,
                                                       const float *__restrict__ w, const uint8_t *__restrict__ issrc,
                                                       Grid g, float prec_dx2)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= g.nx || row >= g.ny) return;
    const int j = row * g.nx + col;
    const size_t N = (size_t)g.N();
    float acc = prec_dx2;
    if (MODE != 3 && row > 0 && row < g.ny - 1 && col > 0 && col < g.nx - 1) {
        const int nx = g.nx;
        if (issrc[j - nx]) acc = __fadd_rn(acc, __fmul_rn(w[3 * N + j - nx], Q[j - nx]));
        if (issrc[j - 1]) acc = __fadd_rn(acc, __fmul_rn(w[2 * N + j - 1], Q[j - 1]));
        if (issrc[j + 1]) acc = __fadd_rn(acc, __fmul_rn(w[1 * N + j + 1], Q[j + 1]));
        if (issrc[j + nx]) acc = __fadd_rn(acc, __fmul_rn(w[j + nx], Q[j + nx]));
        Qn[j] = acc;
        return;
    }
    int c[8];
    const int n = donor_candidates(g, j, row, col, c);
    for (int a = 0; a < n; ++a) {
        const int i = c[a];
        if (!issrc[i]) continue;
        const float qi = Q[i];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (neighbour_i<MODE>(g, i, k) == j) acc = __fadd_rn(acc, __fmul_rn(w[k * N + i], qi));
    }
    Qn[j] = acc;
}

// ---- diffusion, all sweeps in one pass (boundary modes 0-2) -----------------------
// A 64 x 32 tile (512 threads) with a halo of H = nsweeps cells: sweep s is valid on the region
// shrunk by s, so after H sweeps the tile itself is exact.  Per block: zh over the
// region and one more ring (the weights of the region's cells need their
// neighbours), then each region cell's four outgoing weights and source flag
// computed with the weight kernel's operations, then the sweeps on a shrinking
// band, double-buffered in shared memory.  Traffic: zh and Q over the region once,
// temp once.
//
// Periodic modes load the halo with wrap-around, so in modes 0-2 (nx, ny >= 3) the
// k-th neighbour of a cell is always the adjacent shared-memory cell, and it exists
// exactly when that cell lies in the grid along the non-periodic axes.  A cell that
// cannot leave the domain has all four neighbours.  The sources of a cell are
// gathered in ascending global index (the serial order of the reference's atomics):
// top, left, right, bottom, except at the wrapped edges -- periodic EW columns 0 and
// nx-1: top, right, left, bottom; periodic NS row 0: left, right, bottom, top; row
// ny-1: bottom, top, left, right.  Flag byte per region cell: bit 0 in the grid,
// bit 1 a source, bits 2-3 that order.
constexpr int DF_TX = 64, DF_TY = 32, DF_HMAX = 8, DF_THREADS = 512;
__host__ __device__ constexpr int df_region(int H) { return (DF_TX + 2 * H) * (DF_TY + 2 * H); }
__host__ __device__ constexpr int df_ring(int H) { return (DF_TX + 2 * H + 2) * (DF_TY + 2 * H + 2); }
// zh over the region and its ring, four weight planes, two Q buffers, the flags
constexpr size_t df_smem(int H) { return sizeof(float) * (size_t)(df_ring(H) + 6 * df_region(H)) + df_region(H); }

template <int MODE>
__device__ __forceinline__ bool df_inside(const Grid &g, int r, int c)
{
    return (MODE == 2 || (r >= 0 && r < g.ny)) && (MODE == 1 || (c >= 0 && c < g.nx));
}
__device__ __forceinline__ int df_wrap(int v, int n) { return (v >= 0 && v < n) ? v : ((v % n) + n) % n; }


// The weight stored for a link whose source is not a source cell (a boundary cell,
// one outside the domain, or one with sums == 0): real weights are >= 0 or NaN.
constexpr float DF_SKIP = -1.0f;
__device__ __forceinline__ float df_add(float acc, float w, float q)
{
    const float t = __fadd_rn(acc, __fmul_rn(w, q));
    return w != DF_SKIP ? t : acc;
}

template <int MODE, int H>
__global__ void __launch_bounds__(DF_THREADS) k_diffuse_fused(const float *__restrict__ zh, const float *__restrict__ Qin,
                                                       float *__restrict__ out, Grid g, DivC dc, float prec_dx2)
{
    constexpr int RX = DF_TX + 2 * H, RY = DF_TY + 2 * H, ZX = RX + 2, ZY = RY + 2, P = RX * RY;
    extern __shared__ __align__(16) float df_sm[];
    float *zs = df_sm;
    float *w0 = zs + ZX * ZY, *w1 = w0 + P, *w2 = w1 + P, *w3 = w2 + P;
    float *qa = w3 + P, *qb = qa + P;
    unsigned char *fl = reinterpret_cast<unsigned char *>(qb + P);
    const int x0 = blockIdx.x * DF_TX - H, y0 = blockIdx.y * DF_TY - H;  // region origin (unwrapped)
    const int nx = g.nx, ny = g.ny;
    // the region and its ring strictly inside the grid: every region cell is an interior
    // cell (all four neighbours, none on the edge), no wrapping, no domain checks
    const bool inner = x0 >= 1 && y0 >= 1 && x0 + RX < nx && y0 + RY < ny;
    if (inner) {
        for (int t = threadIdx.x; t < ZX * ZY; t += blockDim.x)
            zs[t] = zh[(size_t)(y0 - 1 + t / ZX) * nx + x0 - 1 + t % ZX];
    } else {
        for (int t = threadIdx.x; t < ZX * ZY; t += blockDim.x) {
            const int r = y0 - 1 + t / ZX, c = x0 - 1 + t % ZX;
            zs[t] = df_inside<MODE>(g, r, c) ? zh[df_wrap(r, ny) * nx + df_wrap(c, nx)] : 0.f;
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < P; t += blockDim.x) {
        const int ry = t / RX, rx = t % RX, r = y0 + ry, c = x0 + rx;
        unsigned char f = 0;
        float q = 0.f, wk[4] = {DF_SKIP, DF_SKIP, DF_SKIP, DF_SKIP};
        if (inner || df_inside<MODE>(g, r, c)) {
            const int row = inner ? r : df_wrap(r, ny), col = inner ? c : df_wrap(c, nx);
            q = Qin[row * nx + col];
            f = 1;
            bool leave = false;
            if (!inner) {
                const bool redge = row == 0 || row == ny - 1, cedge = col == 0 || col == nx - 1;
                if (MODE == 1 && cedge) f |= 1 << 2;
                if (MODE == 2 && redge) f |= (row == 0 ? 2 : 3) << 2;
                leave = MODE == 0 ? (redge || cedge) : (MODE == 1 ? redge : cedge);
            }
            if (!leave) {  // all four neighbours exist
                const int z = (ry + 1) * ZX + rx + 1;
                const float zi = zs[z];
                const float zn[4] = {zs[z - ZX], zs[z - 1], zs[z + 1], zs[z + ZX]};
                float sk[4], sums = 0.f;
                // max(0, (zi - zj) / dx) is +0 unless zi > zj (NaN compares false and
                // max(0, NaN) is 0), and 0 / sums is +0 for the sums > 0 of a source:
                // only the descending links divide
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    sk[k] = zi > zn[k] ? fmaxf(0.f, div_dx(__fsub_rn(zi, zn[k]), dc)) : 0.f;
                    sums = __fadd_rn(sums, sk[k]);
                }
                if (sums != 0.f) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) wk[k] = sk[k] != 0.f ? __fdiv_rn(sk[k], sums) : 0.f;
                }
            }
        }
        w0[t] = wk[0];
        w1[t] = wk[1];
        w2[t] = wk[2];
        w3[t] = wk[3];
        qa[t] = q;
        fl[t] = f;
    }
    __syncthreads();
    float *qc = qa, *qn = qb;
#pragma unroll
    for (int sw = 1; sw <= H; ++sw) {
        const int bw = RX - 2 * sw, bh = RY - 2 * sw;
        if (inner) {  // every cell inside the grid, off its edges: summation order top, left, right, bottom
            for (int t = threadIdx.x; t < bw * bh; t += blockDim.x) {
                const int i = (sw + t / bw) * RX + sw + t % bw;
                const int u = i - RX, l = i - 1, rt = i + 1, d = i + RX;
                float acc = prec_dx2;
                acc = df_add(acc, w3[u], qc[u]);
                acc = df_add(acc, w2[l], qc[l]);
                acc = df_add(acc, w1[rt], qc[rt]);
                acc = df_add(acc, w0[d], qc[d]);
                qn[i] = acc;
            }
            __syncthreads();
            float *tq = qc;
            qc = qn;
            qn = tq;
            continue;
        }
        for (int t = threadIdx.x; t < bw * bh; t += blockDim.x) {
            const int i = (sw + t / bw) * RX + sw + t % bw;
            const unsigned char f = fl[i];
            if (!(f & 1)) continue;
            // the source above reaches i through its bottom link (w3), the left one
            // through its right link (w2), the right one its left (w1), below its top (w0);
            // a neighbour that is not a source has the weight DF_SKIP on every link
            const int u = i - RX, l = i - 1, rt = i + 1, d = i + RX;
            float acc = prec_dx2;
            switch (f >> 2) {
            case 0:
                acc = df_add(acc, w3[u], qc[u]);
                acc = df_add(acc, w2[l], qc[l]);
                acc = df_add(acc, w1[rt], qc[rt]);
                acc = df_add(acc, w0[d], qc[d]);
                break;
            case 1:
                acc = df_add(acc, w3[u], qc[u]);
                acc = df_add(acc, w1[rt], qc[rt]);
                acc = df_add(acc, w2[l], qc[l]);
                acc = df_add(acc, w0[d], qc[d]);
                break;
            case 2:
                acc = df_add(acc, w2[l], qc[l]);
                acc = df_add(acc, w1[rt], qc[rt]);
                acc = df_add(acc, w0[d], qc[d]);
                acc = df_add(acc, w3[u], qc[u]);
                break;
            default:
                acc = df_add(acc, w0[d], qc[d]);
                acc = df_add(acc, w3[u], qc[u]);
                acc = df_add(acc, w2[l], qc[l]);
                acc = df_add(acc, w1[rt], qc[rt]);
                break;
            }
            qn[i] = acc;
        }
        __syncthreads();
        float *tq = qc;
        qc = qn;
        qn = tq;
    }
    for (int t = threadIdx.x; t < DF_TX * DF_TY; t += blockDim.x) {
        const int ly = t / DF_TX, lx = t % DF_TX;
        const int row = y0 + H + ly, col = x0 + H + lx;
        if (row < ny && col < nx) out[row * nx + col] = qc[(H + ly) * RX + H + lx];
    }
}

template <int MODE, int H>
static int l_diffuse_fused_h(const float *zh, float *Q, float *temp, const Grid &g, float dx, float prec_dx2,
                             cudaStream_t st)
{
    PFF_CUDA(cudaFuncSetAttribute(k_diffuse_fused<MODE, H>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)df_smem(H)));
    dim3 gr(div_up(g.nx, DF_TX), div_up(g.ny, DF_TY));
    PFF_PROBED("k_diffuse_fused", st,
               k_diffuse_fused<MODE, H><<<gr, DF_THREADS, df_smem(H), st>>>(zh, Q, temp, g, make_divc(dx), prec_dx2));
    count_launch();
    return PFF_OK;
}

template <int MODE>
static int l_diffuse_fused(const float *zh, float *Q, float *temp, int nsweeps, const Grid &g, float dx,
                           float prec_dx2, cudaStream_t st)
{
    switch (nsweeps) {
    case 1: return l_diffuse_fused_h<MODE, 1>(zh, Q, temp, g, dx, prec_dx2, st);
    case 2: return l_diffuse_fused_h<MODE, 2>(zh, Q, temp, g, dx, prec_dx2, st);
    case 3: return l_diffuse_fused_h<MODE, 3>(zh, Q, temp, g, dx, prec_dx2, st);
    case 4: return l_diffuse_fused_h<MODE, 4>(zh, Q, temp, g, dx, prec_dx2, st);
    case 5: return l_diffuse_fused_h<MODE, 5>(zh, Q, temp, g, dx, prec_dx2, st);
    case 6: return l_diffuse_fused_h<MODE, 6>(zh, Q, temp, g, dx, prec_dx2, st);
    case 7: return l_diffuse_fused_h<MODE, 7>(zh, Q, temp, g, dx, prec_dx2, st);
    default: return l_diffuse_fused_h<MODE, 8>(zh, Q, temp, g, dx, prec_dx2, st);
    }
}

// ---- Manning update (gf_hydrodynamics.py:79-129) ------------------------------
// h^(5/3) with the exponent rounded to f32 (Taichi folds 5./3. to an f32
// constant), evaluated in double and rounded once: the correctly rounded f32
// power.  Both the oracle and this kernel use this definition.
__device__ __forceinline__ float pow53(float h) { return (float)pow((double)h, (double)(5.0f / 3.0f)); }

__global__ void __launch_bounds__(256) k_core1(float *h, const float *__restrict__ zh, float *dh,
                                               const int32_t *__restrict__ rec, const float *__restrict__ Q, int N,
                                               float dx, float dx2, float manning, float edgesw, float dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int r = rec[i];
    if ((unsigned)r >= (unsigned)N) r = i;  // an out-of-range receiver reads nothing: the edge slope
    float tS = edgesw;
    if (r != i) tS = fmaxf(__fdiv_rn(__fsub_rn(zh[i], zh[r]), dx), 1e-4f);
    float Qo = __fmul_rn(dx, pow53(h[i]));
    Qo = __fdiv_rn(Qo, manning);
    Qo = __fmul_rn(Qo, __fsqrt_rn(tS));
    float tdh = __fdiv_rn(__fsub_rn(Q[i], Qo), dx2);
    tdh = __fmul_rn(tdh, dt);
    const float h1 = __fadd_rn(h[i], tdh);
    h[i] = h1;
    if (h1 < 0.f) tdh = __fadd_rn(tdh, h1);
    dh[i] = tdh;
}

__global__ void __launch_bounds__(256) k_core2(float *h, float *zh, const float *__restrict__ dh,
                                               const float *__restrict__ href, float *dhmax, int N)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.f;
    if (i < N) {
        const float d = dh[i];
        const float hn = __fadd_rn(h[i], d);
        h[i] = hn;
        zh[i] = __fadd_rn(zh[i], d);
        if (dhmax && href) m = fabsf(__fsub_rn(hn, href[i]));
    }
    if (!dhmax || !href) return;
    // |dh| >= 0 or NaN: as unsigned bits, NaN sorts above every finite value;
    // warp max, block max, then one atomic per block
    unsigned mu = __float_as_uint(m);
    for (int o = 16; o; o >>= 1) mu = max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    __shared__ unsigned wm[8];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mu;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) b = max(b, wm[k]);
        if (b) atomicMax(reinterpret_cast<unsigned int *>(dhmax), b);
    }
}

// Both Manning loops in one pass, for a caller whose zf holds a copy of zh (the
// filled surface the fill leaves in z_ and in zh): the slope reads zf, which no
// thread writes, so zh can be updated in the same pass.  Per cell the operations
// of k_core1 then k_core2, in their order.
__global__ void __launch_bounds__(256) k_core_fused(float *h, float *zh, const float *__restrict__ zf, float *dh,
                                                    const int32_t *__restrict__ rec, const float *__restrict__ Q,
                                                    int N, float dx, float dx2, float manning, float edgesw, float dt,
                                                    const float *__restrict__ href, float *dhmax)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float m = 0.f;
    if (i < N) {
        int r = rec[i];
        if ((unsigned)r >= (unsigned)N) r = i;  // as in k_core1
        const float zi = zf[i];
        float tS = edgesw;
        if (r != i) tS = fmaxf(__fdiv_rn(__fsub_rn(zi, zf[r]), dx), 1e-4f);
        const float hi = h[i];
        float Qo = __fmul_rn(dx, pow53(hi));
        Qo = __fdiv_rn(Qo, manning);
        Qo = __fmul_rn(Qo, __fsqrt_rn(tS));
        float tdh = __fdiv_rn(__fsub_rn(Q[i], Qo), dx2);
        tdh = __fmul_rn(tdh, dt);
        const float h1 = __fadd_rn(hi, tdh);
        if (h1 < 0.f) tdh = __fadd_rn(tdh, h1);
        dh[i] = tdh;
        const float hn = __fadd_rn(h1, tdh);  // k_core2
        h[i] = hn;
        zh[i] = __fadd_rn(zi, tdh);
        if (dhmax && href) m = fabsf(__fsub_rn(hn, href[i]));
    }
    if (!dhmax || !href) return;
    unsigned mu = __float_as_uint(m);
    for (int o = 16; o; o >>= 1) mu = max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    __shared__ unsigned wm[8];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = mu;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned b = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) b = max(b, wm[k]);
        if (b) atomicMax(reinterpret_cast<unsigned int *>(dhmax), b);
    }
}

// out[0] = max |a - b| (as unsigned bits: NaN above every finite value), out[1] += sum |a - b|
__global__ void __launch_bounds__(256) k_abs_diff_stats(const float *__restrict__ a, const float *__restrict__ b, int N,
                                                        float *out)
{
    unsigned mu = 0;
    float s = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const float d = fabsf(__fsub_rn(a[i], b[i]));
        mu = max(mu, __float_as_uint(d));
        s += d;
    }
    for (int o = 16; o; o >>= 1) {
        mu = max(mu, __shfl_xor_sync(0xffffffffu, mu, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mu) atomicMax(reinterpret_cast<unsigned int *>(out), mu);
        atomicAdd(out + 1, s);
    }
}

template <int MODE>
static void l_diffuse(const float *zh, float *Q, float *temp, float *w, uint8_t *issrc, int nsweeps,
                      const Grid &g, float dx, float prec_dx2, cudaStream_t st)
{
    dim3 b(32, 8), gr(div_up(g.nx, 32), div_up(g.ny, 8));
    { k_diffuse_weights<MODE><<<gr, b, 0, st>>>(zh, w, issrc, g, dx); count_launch(); }
    float *a = Q, *c = temp;
    for (int s = 0; s < nsweeps; ++s) {
        { k_diffuse_sweep<MODE><<<gr, b, 0, st>>>(a, c, w, issrc, g, prec_dx2); count_launch(); }
        float *t = a; a = c; c = t;
    }
}

}  // namespace pff

using namespace pff;

static bool g_diffuse_unfused = getenv("PFF_DIFFUSE_UNFUSED") != nullptr;  // diagnostics: the per-sweep kernels

extern "C" size_t pff_fill_workspace_bytes(int N)
{
    if (N < 1) return 256;
    return 2 * Carver::round(sizeof(uint2) * (size_t)N) + Carver::round(sizeof(int) * FILL_FLAGS);
}

// ceil(log2 N) rounds (:121) of the packed fill; `inc(it)` is round it's increment.
// Returns the buffer holding the last round's records.
template <class Inc>
static uint2 *fill_rounds(const float *zh, const int32_t *receivers, void *workspace, size_t workspace_bytes, int N,
                          Inc inc, cudaStream_t st)
{
    Carver cv(workspace, workspace_bytes);
    uint2 *a = cv.take<uint2>(N), *b = cv.take<uint2>(N);
    int *flags = cv.take<int>(FILL_FLAGS);
    { k_fill_pack<<<div_up(N, 256), 256, 0, st>>>(zh, receivers, a, N, flags); count_launch(); }  // :116-117
    int nr = 0;
    for (long long p = 1; p < N; p <<= 1) ++nr;
    int late_blocks = 0;
    if (nr > FILL_VOTE0) {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        late_blocks = std::min(div_up(N, 256 * FILL_CPT), 8 * sms);
    }
    for (int it = 0; it < nr; ++it) {
        if (it < FILL_VOTE0) {
            PFF_PROBED("k_fill_round_packed", st,
                       k_fill_round_packed<<<div_up(N, 256 * FILL_CPT), 256, 0, st>>>(zh, a, b, inc(it), N));
        } else {
            PFF_PROBED("k_fill_round_late", st,
                       k_fill_round_late<<<late_blocks, 256, 0, st>>>(zh, a, b, inc(it), N, flags, it));
        }
        count_launch();
        std::swap(a, b);
    }
    return a;
}

extern "C" int pff_fill_z_add_delta(float *zh, float *h, float *z_, const int32_t *receivers, int32_t *receivers_,
                                    int32_t *receivers__, double epsilon, int N, void *workspace,
                                    size_t workspace_bytes, void *stream)
{
    clear_error();
    if (N <= 1 || !zh || !h || !z_ || !receivers || !receivers_ || !receivers__) {
        set_error("pff_fill_z_add_delta: bad arguments");
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_fill_workspace_bytes(N)) {
        set_error("pff_fill_z_add_delta: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    // Python folds 2**(it-1)*eps in double
    const uint2 *a = fill_rounds(zh, receivers, workspace, workspace_bytes, N,
                                 [&](int it) { return (float)(ldexp(1.0, it - 1) * epsilon); }, st);
    { k_fill_unpack<<<div_up(N, 256), 256, 0, st>>>(a, z_, receivers_, receivers__, zh, h, false, N); count_launch(); }
    return check_cuda("pff_fill_z_add_delta");
}

// ---- fill without caller-provided scratch -----------------------------------------
//
// For callers that cannot allocate device memory (for example code running
// under an allocator that forbids new allocations, or a host that only hands
// out the buffers it owns): the one scratch buffer of the fill -- the
// start-of-round snapshot of z_ -- lives in this file-scope device array
// instead of a workspace.  It holds PFF_NOALLOC_MAX_CELLS floats (16 MiB) on
// every GPU that loads the library, until the process exits.
static __device__ __align__(256) float g_fill_scratch[PFF_NOALLOC_MAX_CELLS];

// Device address of g_fill_scratch per device, looked up once with that device
// current (the host-side symbol is only a stand-in, not a device address).
// Atomic entries: host threads may make their first call concurrently; each
// looks up the same address, so whichever store lands is correct.  The cached
// address belongs to the device's current context: after cudaDeviceReset the
// library's module is loaded again and the cache must not be trusted, so a
// process that resets a device does not use this entry point afterwards.
static std::atomic<float *> g_fill_scratch_ptr[64];

static int fill_scratch_address(float **out)
{
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("pff_fill_z_add_delta_noalloc: device index %d out of range", dev);
        return PFF_ERR_ARG;
    }
    float *ptr = g_fill_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!ptr) {
        void *p = nullptr;
        PFF_CUDA(cudaGetSymbolAddress(&p, g_fill_scratch));
        ptr = (float *)p;
        g_fill_scratch_ptr[dev].store(ptr, std::memory_order_release);
    }
    *out = ptr;
    return PFF_OK;
}

extern "C" int pff_fill_z_add_delta_noalloc(float *zh, float *h, float *z_, const int32_t *receivers,
                                            int32_t *receivers_, int32_t *receivers__, double epsilon, int N,
                                            void *stream)
{
    clear_error();
    if (N <= 1 || !zh || !h || !z_ || !receivers || !receivers_ || !receivers__) {
        set_error("pff_fill_z_add_delta_noalloc: bad arguments");
        return PFF_ERR_ARG;
    }
    if (N > PFF_NOALLOC_MAX_CELLS) {
        set_error("pff_fill_z_add_delta_noalloc: %d cells exceed the built-in scratch of %d cells; "
                  "use pff_fill_z_add_delta with a workspace",
                  N, PFF_NOALLOC_MAX_CELLS);
        return PFF_ERR_ARG;
    }
    float *zt = nullptr;
    PFF_TRY(fill_scratch_address(&zt));
    cudaStream_t st = S(stream);
    const size_t nbf = sizeof(float) * (size_t)N, nbi = sizeof(int32_t) * (size_t)N;
    PFF_CUDA(cudaMemcpyAsync(z_, zh, nbf, cudaMemcpyDeviceToDevice, st));
    PFF_CUDA(cudaMemcpyAsync(receivers_, receivers, nbi, cudaMemcpyDeviceToDevice, st));
    int nr = 0;
    for (long long p = 1; p < N; p <<= 1) ++nr;
    // every round writes all N snapshot entries before any is read: nothing to clear
    float *zs = z_, *zn = zt;
    int32_t *ra = receivers_, *rb = receivers__;
    for (int it = 0; it < nr; ++it) {
        const float inc = (float)(ldexp(1.0, it - 1) * epsilon);
        { k_fill_round<<<div_up(N, 256), 256, 0, st>>>(zh, zs, zn, ra, rb, inc, N); count_launch(); }
        float *tz = zs; zs = zn; zn = tz;
        int32_t *tr = ra; ra = rb; rb = tr;
    }
    if (zs != z_) PFF_CUDA(cudaMemcpyAsync(z_, zs, nbf, cudaMemcpyDeviceToDevice, st));
    PFF_CUDA(cudaMemcpyAsync(rb, ra, nbi, cudaMemcpyDeviceToDevice, st));
    { k_fill_apply<<<div_up(N, 256), 256, 0, st>>>(zh, h, z_, N); count_launch(); }
    return check_cuda("pff_fill_z_add_delta_noalloc");
}

// topofill (fill_topo.py:48-78 driving _topofill :17-45): the same pointer-jumping
// rounds with increments 2^it * epsilon for it = 0..ceil(log2 N)-1 (the reference
// passes iteration it+1 and uses 2^(iteration-1)), then z = z_; no depth update.
extern "C" int pff_topofill(float *z, float *z_, const int32_t *receivers, int32_t *receivers_, int32_t *receivers__,
                            double epsilon, int N, int write_back, void *workspace, size_t workspace_bytes,
                            void *stream)
{
    clear_error();
    if (N <= 1 || !z || !z_ || !receivers || !receivers_ || !receivers__) {
        set_error("pff_topofill: bad arguments");
        return PFF_ERR_ARG;
    }
    if (!workspace || workspace_bytes < pff_fill_workspace_bytes(N)) {
        set_error("pff_topofill: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    cudaStream_t st = S(stream);
    // 2^it * float(epsilon): a power-of-2 scaling
    const uint2 *a = fill_rounds(z, receivers, workspace, workspace_bytes, N,
                                 [&](int it) { return (float)(ldexp(1.0, it) * epsilon); }, st);
    { k_fill_unpack<<<div_up(N, 256), 256, 0, st>>>(a, z_, receivers_, receivers__, z, nullptr, write_back != 0, N);
      count_launch(); }
    return check_cuda("pff_topofill");
}

extern "C" size_t pff_diffuse_workspace_bytes(int N)
{
    return Carver::round(sizeof(float) * 4 * (size_t)N) + Carver::round((size_t)N) + 512;
}

extern "C" int pff_diffuse_q(const float *zh, float *Q, float *temp, int nsweeps, int nx, int ny, float dx,
                             float prec_dx2, int bound_mode, const uint8_t *codes, void *workspace,
                             size_t workspace_bytes, void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!zh || !Q || !temp || nsweeps < 0) { set_error("pff_diffuse_q: bad arguments"); return PFF_ERR_ARG; }
    const int N = nx * ny;
    if (!workspace || workspace_bytes < pff_diffuse_workspace_bytes(N)) {
        set_error("pff_diffuse_q: workspace too small");
        return PFF_ERR_WORKSPACE;
    }
    if (nsweeps == 0) return PFF_OK;
    Grid g{nx, ny, bound_mode, codes};
    cudaStream_t st = S(stream);
    if (bound_mode != 3 && nx >= 3 && ny >= 3 && nsweeps <= DF_HMAX && !g_diffuse_unfused) {
        // every sweep in one pass into temp (Q is read as other tiles' halo), then Q = temp (:74-75)
        int rc = PFF_OK;
        switch (bound_mode) {
        case 0: rc = l_diffuse_fused<0>(zh, Q, temp, nsweeps, g, dx, prec_dx2, st); break;
        case 1: rc = l_diffuse_fused<1>(zh, Q, temp, nsweeps, g, dx, prec_dx2, st); break;
        default: rc = l_diffuse_fused<2>(zh, Q, temp, nsweeps, g, dx, prec_dx2, st); break;
        }
        PFF_TRY(rc);
        PFF_CUDA(cudaMemcpyAsync(Q, temp, sizeof(float) * (size_t)N, cudaMemcpyDeviceToDevice, st));
        return check_cuda("pff_diffuse_q");
    }
    Carver cv(workspace, workspace_bytes);
    float *w = cv.take<float>(4 * (size_t)N);
    uint8_t *issrc = cv.take<uint8_t>(N);
    PFF_MODE_DISPATCH(bound_mode, l_diffuse, zh, Q, temp, w, issrc, nsweeps, g, dx, prec_dx2, st);
    // the reference ends each sweep with Q == temp (:74-75)
    const size_t nbf = sizeof(float) * (size_t)N;
    if (nsweeps & 1) PFF_CUDA(cudaMemcpyAsync(Q, temp, nbf, cudaMemcpyDeviceToDevice, st));
    else PFF_CUDA(cudaMemcpyAsync(temp, Q, nbf, cudaMemcpyDeviceToDevice, st));
    return check_cuda("pff_diffuse_q");
}

extern "C" int pff_graphflood_core(float *h, float *zh, float *dh, const int32_t *rec, const float *Q, int N,
                                   float dx, float dx2, float manning, float edgesw, float dt, const float *h_ref,
                                   float *dhmax, void *stream)
{
    clear_error();
    if (N <= 0 || !h || !zh || !dh || !rec || !Q) { set_error("pff_graphflood_core: bad arguments"); return PFF_ERR_ARG; }
    cudaStream_t st = S(stream);
    { k_core1<<<div_up(N, 256), 256, 0, st>>>(h, zh, dh, rec, Q, N, dx, dx2, manning, edgesw, dt); count_launch(); }
    { k_core2<<<div_up(N, 256), 256, 0, st>>>(h, zh, dh, h_ref, dhmax, N); count_launch(); }
    return check_cuda("pff_graphflood_core");
}

extern "C" int pff_graphflood_core_filled(float *h, float *zh, const float *zf, float *dh, const int32_t *rec,
                                          const float *Q, int N, float dx, float dx2, float manning, float edgesw,
                                          float dt, const float *h_ref, float *dhmax, void *stream)
{
    clear_error();
    if (N <= 0 || !h || !zh || !zf || !dh || !rec || !Q || zf == zh) {
        set_error("pff_graphflood_core_filled: bad arguments");
        return PFF_ERR_ARG;
    }
    cudaStream_t st = S(stream);
    PFF_PROBED("k_core_fused", st,
               k_core_fused<<<div_up(N, 256), 256, 0, st>>>(h, zh, zf, dh, rec, Q, N, dx, dx2, manning, edgesw, dt,
                                                             h_ref, dhmax));
    count_launch();
    return check_cuda("pff_graphflood_core_filled");
}

extern "C" int pff_abs_diff_stats(const float *a, const float *b, int N, float *out, void *stream)
{
    clear_error();
    if (!a || !b || !out || N <= 0) { set_error("pff_abs_diff_stats: bad arguments"); return PFF_ERR_ARG; }
    const int blocks = std::min(div_up(N, 256), 148 * 8);
    { k_abs_diff_stats<<<blocks, 256, 0, S(stream)>>>(a, b, N, out); count_launch(); }
    return check_cuda("pff_abs_diff_stats");
}
