// libpff convolutions for the GraphFlood warm-start network: BF16 3x3 convolution
// (stride 1, zero padding 1) as an implicit GEMM on the tensor cores with FP32
// accumulation -- forward, data gradient (the forward kernel on flipped,
// transposed weights) and weight gradient -- plus the small ops of a U-Net
// (2x2 average pooling, nearest 2x upsampling into a concatenation slice, ReLU
// backward, bias gradient, masked MSE loss, Adam).  No reference counterpart:
// the reference has no learned component.
//
// Activations are NHWC bf16 rows of `cs` channels; an operand may be a channel
// slice [off, off + C) of a wider row (the U-Net's concatenations), so every
// tensor argument is (pointer, row stride cs, channel offset off).  Weights are
// [Cout][9][Cin] bf16 (k = tap*Cin + ci, tap = kh*3 + kw).
//
// GEMM mapping (forward): M = pixels, N = Cout, K = 9*Cin.  A rows are gathered
// 16 bytes at a time straight from the activations with zero fill for the halo
// (cp.async, 3-stage pipeline), fragments come from XOR-swizzled shared memory
// through ldmatrix, products are mma.sync m16n8k16 bf16 -> f32.
#include <cuda_bf16.h>
#include "pff_internal.h"

namespace pff {

typedef uint16_t bf16_t;  // raw bf16 bits in the C ABI

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(unsigned dst, const void *src, bool valid)
{
    const int n = valid ? 16 : 0;  // 0 source bytes: the 16 destination bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(unsigned addr, unsigned &r0, unsigned &r1, unsigned &r2, unsigned &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void mma16816(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3, unsigned b0,
                                         unsigned b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float bf2f(bf16_t v) { return __uint_as_float((unsigned)v << 16); }
__device__ __forceinline__ bf16_t f2bf(float f)
{
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<bf16_t *>(&b);
}

// ---- forward / data-gradient convolution ---------------------------------------------
constexpr int CV_BM = 128, CV_BN = 64, CV_BK = 32, CV_ST = 3, CV_THREADS = 128;

struct ConvArgs {
    const bf16_t *x;
    int csx, offx;
    const bf16_t *w;  // [Cout][9*Cin]
    const float *bias;
    void *y;
    int csy, offy;
    int B, H, W, Cin, Cout;
    int relu, out_f32;
};

// 64-byte rows (4 chunks of 16 B), chunk c of row r stored at c ^ ((r >> 1) & 3)
__device__ __forceinline__ int sw64(int r, int c) { return r * 4 + (c ^ ((r >> 1) & 3)); }

__global__ void __launch_bounds__(CV_THREADS) k_conv3x3(ConvArgs a)
{
    __shared__ __align__(128) uint4 sA[CV_ST][CV_BM * 4];
    __shared__ __align__(128) uint4 sB[CV_ST][CV_BN * 4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const long long P = (long long)a.B * a.H * a.W;
    const long long m0 = (long long)blockIdx.x * CV_BM;
    const int n0 = blockIdx.y * CV_BN;
    const int K = 9 * a.Cin;
    const int nk = (K + CV_BK - 1) / CV_BK;

    // this thread's A rows (4) and chunk: rows tid/4 + 32j, chunk tid%4
    const int ac = tid & 3;
    int ay[4], ax[4];
    long long abase[4];
    bool aval[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const long long p = m0 + (tid >> 2) + 32 * j;
        aval[j] = p < P;
        const long long pp = aval[j] ? p : 0;
        const int x = (int)(pp % a.W);
        const long long t = pp / a.W;
        ay[j] = (int)(t % a.H);
        ax[j] = x;
        abase[j] = (t / a.H) * a.H;  // b * H
    }
    // B rows (2): n = tid/4 + 32j, chunk tid%4
    auto load_stage = [&](int st, int kt) {
        const int k = kt * CV_BK + ac * 8;
        const bool kval = k < K;
        const int tap = kval ? k / a.Cin : 0;
        const int ci = kval ? k - tap * a.Cin : 0;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int r = (tid >> 2) + 32 * j;
            const int yy = ay[j] + dy, xx = ax[j] + dx;
            const bool v = kval && aval[j] && yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
            const bf16_t *src = v ? a.x + ((abase[j] + yy) * a.W + xx) * a.csx + a.offx + ci : a.x;
            cp_async16(smem_u32(&sA[st][sw64(r, ac)]), src, v);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int r = (tid >> 2) + 32 * j;
            const int co = n0 + r;
            const bool v = kval && co < a.Cout;
            const bf16_t *src = v ? a.w + (long long)co * K + k : a.w;
            cp_async16(smem_u32(&sB[st][sw64(r, ac)]), src, v);
        }
    };

    float acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;

#pragma unroll
    for (int s = 0; s < CV_ST - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_wait<CV_ST - 2>();
        __syncthreads();
        {  // prefetch stage kt + ST - 1 (its buffer was consumed at iteration kt - 1)
            const int nt = kt + CV_ST - 1;
            if (nt < nk) load_stage(nt % CV_ST, nt);
            cp_commit();
        }
        const int st = kt % CV_ST;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {  // two k16 steps per 32-wide stage
            unsigned af[4][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = wm * 64 + i * 16 + (lane & 15);
                const int c = kk * 2 + (lane >> 4);
                ldsm_x4(smem_u32(&sA[st][sw64(r, c)]), af[i][0], af[i][1], af[i][2], af[i][3]);
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int r = wn * 32 + j * 16 + (lane & 7) + ((lane >> 4) << 3);
                const int c = kk * 2 + ((lane >> 3) & 1);
                unsigned r0, r1, r2, r3;
                ldsm_x4(smem_u32(&sB[st][sw64(r, c)]), r0, r1, r2, r3);
                bfr[2 * j][0] = r0;
                bfr[2 * j][1] = r1;
                bfr[2 * j + 1][0] = r2;
                bfr[2 * j + 1][1] = r3;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mma16816(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bfr[j][0], bfr[j][1]);
        }
    }
    cp_wait<0>();

    // epilogue: bias, ReLU, store (bf16 pairs, or f32)
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const long long p = m0 + wm * 64 + i * 16 + (lane >> 2) + hf * 8;
            if (p >= P) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int co = n0 + wn * 32 + j * 8 + 2 * (lane & 3);
                if (co >= a.Cout) continue;
                float v0 = acc[i][j][2 * hf], v1 = acc[i][j][2 * hf + 1];
                if (a.bias) {
                    v0 += a.bias[co];
                    if (co + 1 < a.Cout) v1 += a.bias[co + 1];
                }
                if (a.relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                if (a.out_f32) {
                    float *yo = (float *)a.y + p * a.csy + a.offy + co;
                    yo[0] = v0;
                    if (co + 1 < a.Cout) yo[1] = v1;
                } else {
                    bf16_t *yo = (bf16_t *)a.y + p * a.csy + a.offy + co;
                    if (co + 1 < a.Cout) {
                        const unsigned pk = (unsigned)f2bf(v0) | ((unsigned)f2bf(v1) << 16);
                        *reinterpret_cast<unsigned *>(yo) = pk;
                    } else {
                        yo[0] = f2bf(v0);
                    }
                }
            }
        }
}

// wt[ci][tap'][co] = w[co][8 - tap'][ci]: the data gradient of a 3x3 convolution is
// the forward convolution of dy with these weights.
__global__ void k_wflip(const bf16_t *__restrict__ w, bf16_t *wt, int Cin, int Cout)
{
    const long long n = 9LL * Cin * Cout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int co = (int)(e % Cout);
        const long long t = e / Cout;
        const int tp = (int)(t % 9);
        const int ci = (int)(t / 9);
        wt[e] = w[((long long)co * 9 + (8 - tp)) * Cin + ci];
    }
}

// ---- weight gradient --------------------------------------------------------------------
// dw[co][k] += sum_p dy[p][co] * x~[p][k],  x~[p][k] = x[shift(p, tap(k))][ci(k)] (0 outside).
// GEMM M = Cout, N = 9*Cin, reduced over pixels; each CTA reduces one pixel range
// and adds its 64 x 64 tile into dw with f32 atomics.
constexpr int WG_BM = 64, WG_BN = 64, WG_BK = 32, WG_ST = 3, WG_THREADS = 128;

struct WgradArgs {
    const bf16_t *x;
    int csx, offx;
    const bf16_t *dy;
    int csd, offd;
    float *dw;
    int B, H, W, Cin, Cout;
    long long pchunk;  // pixels per CTA (multiple of WG_BK)
};

// 128-byte rows (8 chunks), chunk c of row r stored at c ^ (r & 7)
__device__ __forceinline__ int sw128(int r, int c) { return r * 8 + (c ^ (r & 7)); }

__global__ void __launch_bounds__(WG_THREADS) k_conv3x3_wgrad(WgradArgs a)
{
    __shared__ __align__(128) uint4 sA[WG_ST][WG_BK * 8];  // [pixel][co]
    __shared__ __align__(128) uint4 sB[WG_ST][WG_BK * 8];  // [pixel][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp >> 1, wn = warp & 1;
    const long long P = (long long)a.B * a.H * a.W;
    const int K = 9 * a.Cin;
    const int n0 = blockIdx.x * WG_BN, m0 = blockIdx.y * WG_BM;
    const long long pb = (long long)blockIdx.z * a.pchunk;
    const long long pe = min(P, pb + a.pchunk);
    if (pb >= pe) return;
    const int nk = (int)((pe - pb + WG_BK - 1) / WG_BK);
    // loads: rows r = tid/8 + 16j (j = 0, 1), chunk tid%8, for both A and B
    const int lc = tid & 7;
    const int kb = n0 + lc * 8;  // this thread's B column chunk
    const bool kval = kb < K;
    const int tap = kval ? kb / a.Cin : 0;
    const int ci = kval ? kb - tap * a.Cin : 0;
    const int ddy = tap / 3 - 1, ddx = tap % 3 - 1;
    const int coA = m0 + lc * 8;
    const bool cval = coA < a.Cout;
    auto load_stage = [&](int st, int kt) {
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int r = (tid >> 3) + 16 * j;
            const long long p = pb + (long long)kt * WG_BK + r;
            const bool pv = p < pe;
            const bf16_t *srcA = (pv && cval) ? a.dy + p * a.csd + a.offd + coA : a.dy;
            cp_async16(smem_u32(&sA[st][sw128(r, lc)]), srcA, pv && cval);
            bool v = pv && kval;
            const bf16_t *srcB = a.x;
            if (v) {
                const int x = (int)(p % a.W);
                const long long t = p / a.W;
                const int y = (int)(t % a.H);
                const long long b = t / a.H;
                const int yy = y + ddy, xx = x + ddx;
                v = yy >= 0 && yy < a.H && xx >= 0 && xx < a.W;
                if (v) srcB = a.x + ((b * a.H + yy) * a.W + xx) * a.csx + a.offx + ci;
            }
            cp_async16(smem_u32(&sB[st][sw128(r, lc)]), srcB, v);
        }
    };
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.f;
#pragma unroll
    for (int s = 0; s < WG_ST - 1; ++s) {
        if (s < nk) load_stage(s, s);
        cp_commit();
    }
    for (int kt = 0; kt < nk; ++kt) {
        cp_wait<WG_ST - 2>();
        __syncthreads();
        {
            const int nt = kt + WG_ST - 1;
            if (nt < nk) load_stage(nt % WG_ST, nt);
            cp_commit();
        }
        const int st = kt % WG_ST;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            unsigned af[2][4], bfr[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {  // A^T from [pixel][co]: trans loads
                const int r = kk * 16 + (lane & 7) + ((lane >> 4) << 3);
                const int c = (wm * 32 + i * 16) / 8 + ((lane >> 3) & 1);
                ldsm_x4_t(smem_u32(&sA[st][sw128(r, c)]), af[i][0], af[i][1], af[i][2], af[i][3]);
            }
#pragma unroll
            for (int j = 0; j < 2; ++j) {  // B from [pixel][k]: trans loads
                const int r = kk * 16 + (lane & 7) + (((lane >> 3) & 1) << 3);
                const int c = (wn * 32 + j * 16) / 8 + (lane >> 4);
                unsigned r0, r1, r2, r3;
                ldsm_x4_t(smem_u32(&sB[st][sw128(r, c)]), r0, r1, r2, r3);
                bfr[2 * j][0] = r0;
                bfr[2 * j][1] = r1;
                bfr[2 * j + 1][0] = r2;
                bfr[2 * j + 1][1] = r3;
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mma16816(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bfr[j][0], bfr[j][1]);
        }
    }
    cp_wait<0>();
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int hf = 0; hf < 2; ++hf) {
            const int co = m0 + wm * 32 + i * 16 + (lane >> 2) + hf * 8;
            if (co >= a.Cout) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int k = n0 + wn * 32 + j * 8 + 2 * (lane & 3);
                if (k < K) atomicAdd(a.dw + (long long)co * K + k, acc[i][j][2 * hf]);
                if (k + 1 < K) atomicAdd(a.dw + (long long)co * K + k + 1, acc[i][j][2 * hf + 1]);
            }
        }
}

// ---- small ops --------------------------------------------------------------------------
#define GRID_STRIDE(e, n) \
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (n); e += (long long)gridDim.x * blockDim.x)

// db[c] += sum_p dy[p][c]: each block reduces a pixel range per channel
__global__ void k_bias_grad(const bf16_t *__restrict__ dy, int cs, int off, float *db, long long P, int C)
{
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int l = threadIdx.x / C;
    if (l >= lanes) return;
    float s = 0.f;
    for (long long p = blockIdx.x * (long long)lanes + l; p < P; p += (long long)gridDim.x * lanes)
        s += bf2f(dy[p * cs + off + c]);
    atomicAdd(db + c, s);
}

__global__ void k_relu_bwd(bf16_t *g, int csg, int offg, const bf16_t *__restrict__ y, int csy, int offy, long long P,
                           int C)
{
    GRID_STRIDE(e, P * C)
    {
        const long long p = e / C;
        const int c = (int)(e - p * C);
        if (!(bf2f(y[p * csy + offy + c]) > 0.f)) g[p * csg + offg + c] = 0;
    }
}

// y[b, Y, X] = mean of the 2x2 block of x (H, W even: the fine grid)
__global__ void k_avgpool2(const bf16_t *__restrict__ x, int csx, int offx, bf16_t *y, int csy, int offy, int B, int H,
                           int W, int C)
{
    const int h2 = H / 2, w2 = W / 2;
    GRID_STRIDE(e, (long long)B * h2 * w2 * C)
    {
        const int c = (int)(e % C);
        const long long q = e / C;
        const int X = (int)(q % w2);
        const long long t = q / w2;
        const int Y = (int)(t % h2);
        const long long b = t / h2;
        const long long p00 = (b * H + 2 * Y) * W + 2 * X;
        const float s = bf2f(x[p00 * csx + offx + c]) + bf2f(x[(p00 + 1) * csx + offx + c]) +
                        bf2f(x[(p00 + W) * csx + offx + c]) + bf2f(x[(p00 + W + 1) * csx + offx + c]);
        y[q * csy + offy + c] = f2bf(0.25f * s);
    }
}

// dx[fine] (+)= dy[coarse] / 4
__global__ void k_avgpool2_bwd(const bf16_t *__restrict__ dy, int csd, int offd, bf16_t *dx, int csx, int offx, int B,
                               int H, int W, int C, int accumulate)
{
    const int h2 = H / 2, w2 = W / 2;
    GRID_STRIDE(e, (long long)B * H * W * C)
    {
        const int c = (int)(e % C);
        const long long p = e / C;
        const int x = (int)(p % W);
        const long long t = p / W;
        const int y = (int)(t % H);
        const long long b = t / H;
        const long long q = (b * h2 + y / 2) * w2 + x / 2;
        float v = 0.25f * bf2f(dy[q * csd + offd + c]);
        bf16_t *o = dx + p * csx + offx + c;
        if (accumulate) v += bf2f(*o);
        *o = f2bf(v);
    }
}

// y[fine] = x[coarse] (nearest), H, W: the coarse grid
__global__ void k_upsample2(const bf16_t *__restrict__ x, int csx, int offx, bf16_t *y, int csy, int offy, int B, int H,
                            int W, int C)
{
    const int H2 = 2 * H, W2 = 2 * W;
    GRID_STRIDE(e, (long long)B * H2 * W2 * C)
    {
        const int c = (int)(e % C);
        const long long p = e / C;
        const int X = (int)(p % W2);
        const long long t = p / W2;
        const int Y = (int)(t % H2);
        const long long b = t / H2;
        y[p * csy + offy + c] = x[((b * H + Y / 2) * W + X / 2) * csx + offx + c];
    }
}

// dx[coarse] = sum of dy over the 2x2 block
__global__ void k_upsample2_bwd(const bf16_t *__restrict__ dy, int csd, int offd, bf16_t *dx, int csx, int offx, int B,
                                int H, int W, int C)
{
    const int W2 = 2 * W;
    GRID_STRIDE(e, (long long)B * H * W * C)
    {
        const int c = (int)(e % C);
        const long long q = e / C;
        const int X = (int)(q % W);
        const long long t = q / W;
        const int Y = (int)(t % H);
        const long long b = t / H;
        const long long p00 = (b * 2 * H + 2 * Y) * W2 + 2 * X;
        const float s = bf2f(dy[p00 * csd + offd + c]) + bf2f(dy[(p00 + 1) * csd + offd + c]) +
                        bf2f(dy[(p00 + W2) * csd + offd + c]) + bf2f(dy[(p00 + W2 + 1) * csd + offd + c]);
        dx[q * csx + offx + c] = f2bf(s);
    }
}

// loss += sum_p w_p (pred_p - t_p)^2 * scale; dpred[p][0] = 2 w_p (pred_p - t_p) * scale (bf16),
// the other channels of the dpred row zeroed.
__global__ void k_mse(const float *__restrict__ pred, int csp, const float *__restrict__ tgt,
                      const float *__restrict__ wgt, long long P, bf16_t *dpred, int csd, float scale, float *loss)
{
    float s = 0.f;
    GRID_STRIDE(p, P)
    {
        const float w = wgt ? wgt[p] : 1.f;
        const float d = pred[p * csp] - tgt[p];
        s += w * d * d;
        bf16_t *o = dpred + p * csd;
        o[0] = f2bf(2.f * w * d * scale);
        for (int c = 1; c < csd; ++c) o[c] = 0;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * scale);
}

// Adam (decoupled weight decay); writes the bf16 copy of the parameters if asked
__global__ void k_adam(float *p, const float *__restrict__ g, float *m, float *v, bf16_t *pb, long long n, float lr,
                       float b1, float b2, float eps, float bc1, float bc2, float wd)
{
    GRID_STRIDE(e, n)
    {
        const float gi = g[e];
        const float mi = b1 * m[e] + (1.f - b1) * gi;
        const float vi = b2 * v[e] + (1.f - b2) * gi * gi;
        m[e] = mi;
        v[e] = vi;
        float pi = p[e] * (1.f - lr * wd);
        pi -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        p[e] = pi;
        if (pb) pb[e] = f2bf(pi);
    }
}

__global__ void k_f32_to_bf16(const float *__restrict__ s, bf16_t *d, long long n)
{
    GRID_STRIDE(e, n) d[e] = f2bf(s[e]);
}

static int grid_for(long long n, int threads = 256)
{
    long long b = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

// the tcgen05 forward (pff_conv_tc.cu)
int conv_path();
bool conv_tc_supported(int H, int W, int Cin, int Cout, int csx, int offx, int csy, int offy, int out_f32, int *BW,
                       int *BH);
int conv3x3_tc(const bf16_t *x, int csx, int offx, const bf16_t *w, const float *bias, void *y, int csy, int offy,
               int B, int H, int W, int Cin, int Cout, int relu, int out_f32, cudaStream_t st);

static int check_slice(const char *who, int cs, int off, int C)
{
    if (cs <= 0 || off < 0 || C <= 0 || off + C > cs) {
        set_error("%s: channel slice [%d, %d) outside rows of %d", who, off, off + C, cs);
        return PFF_ERR_ARG;
    }
    return PFF_OK;
}

}  // namespace pff

using namespace pff;

extern "C" int pff_conv3x3_fwd(const bf16_t *x, int csx, int offx, const bf16_t *w, const float *bias, void *y,
                               int csy, int offy, int B, int H, int W, int Cin, int Cout, int relu, int out_f32,
                               void *stream)
{
    clear_error();
    if (!x || !w || !y || B <= 0 || H <= 0 || W <= 0 || Cin <= 0 || Cout <= 0 || Cin % 8 || csx % 8 || offx % 8) {
        set_error("pff_conv3x3_fwd: bad arguments (Cin, row stride and offset must be multiples of 8)");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_conv3x3_fwd input", csx, offx, Cin));
    PFF_TRY(check_slice("pff_conv3x3_fwd output", csy, offy, Cout));
    if (!out_f32 && ((Cout % 2 && Cout != 1) || csy % 2 || offy % 2)) {
        set_error("pff_conv3x3_fwd: bf16 output needs even Cout, row stride and offset");
        return PFF_ERR_ARG;
    }
    const int path = conv_path();
    int bw, bh;
    const bool tc_ok = conv_tc_supported(H, W, Cin, Cout, csx, offx, csy, offy, out_f32, &bw, &bh);
    if (path == 2 || (path == 0 && tc_ok))
        return conv3x3_tc(x, csx, offx, w, bias, y, csy, offy, B, H, W, Cin, Cout, relu, out_f32, S(stream));
    ConvArgs a{x, csx, offx, w, bias, y, csy, offy, B, H, W, Cin, Cout, relu, out_f32};
    const long long P = (long long)B * H * W;
    dim3 grid((unsigned)((P + CV_BM - 1) / CV_BM), (unsigned)((Cout + CV_BN - 1) / CV_BN));
    { k_conv3x3<<<grid, CV_THREADS, 0, S(stream)>>>(a); count_launch(); }
    return check_cuda("pff_conv3x3_fwd");
}

extern "C" int pff_conv3x3_wflip(const bf16_t *w, bf16_t *wt, int Cin, int Cout, void *stream)
{
    clear_error();
    if (!w || !wt || Cin <= 0 || Cout <= 0) {
        set_error("pff_conv3x3_wflip: bad arguments");
        return PFF_ERR_ARG;
    }
    const long long n = 9LL * Cin * Cout;
    { k_wflip<<<grid_for(n), 256, 0, S(stream)>>>(w, wt, Cin, Cout); count_launch(); }
    return check_cuda("pff_conv3x3_wflip");
}

extern "C" int pff_conv3x3_wgrad(const bf16_t *x, int csx, int offx, const bf16_t *dy, int csd, int offd, float *dw,
                                 int B, int H, int W, int Cin, int Cout, void *stream)
{
    clear_error();
    if (!x || !dy || !dw || B <= 0 || H <= 0 || W <= 0 || Cin % 8 || Cout % 8 || Cin <= 0 || Cout <= 0 || csx % 8 ||
        offx % 8 || csd % 8 || offd % 8) {
        set_error("pff_conv3x3_wgrad: bad arguments (channels, strides, offsets multiples of 8)");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_conv3x3_wgrad input", csx, offx, Cin));
    PFF_TRY(check_slice("pff_conv3x3_wgrad dy", csd, offd, Cout));
    const long long P = (long long)B * H * W;
    const int K = 9 * Cin;
    const int tiles = ((K + WG_BN - 1) / WG_BN) * ((Cout + WG_BM - 1) / WG_BM);
    // enough pixel chunks for ~4 CTAs per SM, each at least 512 pixels
    long long chunks = std::max<long long>(1, (148LL * 4 + tiles - 1) / tiles);
    long long pchunk = (P + chunks - 1) / chunks;
    pchunk = std::max<long long>(512, (pchunk + WG_BK - 1) / WG_BK * WG_BK);
    chunks = (P + pchunk - 1) / pchunk;
    WgradArgs a{x, csx, offx, dy, csd, offd, dw, B, H, W, Cin, Cout, pchunk};
    dim3 grid((unsigned)((K + WG_BN - 1) / WG_BN), (unsigned)((Cout + WG_BM - 1) / WG_BM), (unsigned)chunks);
    { k_conv3x3_wgrad<<<grid, WG_THREADS, 0, S(stream)>>>(a); count_launch(); }
    return check_cuda("pff_conv3x3_wgrad");
}

extern "C" int pff_bias_grad(const bf16_t *dy, int cs, int off, float *db, long long P, int C, void *stream)
{
    clear_error();
    if (!dy || !db || P <= 0 || C <= 0 || C > 256) {
        set_error("pff_bias_grad: bad arguments (1 <= C <= 256)");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_bias_grad", cs, off, C));
    const int lanes = std::max(1, 256 / C);
    const int blocks = (int)std::min<long long>(1184, (P + lanes - 1) / lanes);
    { k_bias_grad<<<blocks, lanes * C, 0, S(stream)>>>(dy, cs, off, db, P, C); count_launch(); }
    return check_cuda("pff_bias_grad");
}

extern "C" int pff_relu_bwd(bf16_t *g, int csg, int offg, const bf16_t *y, int csy, int offy, long long P, int C,
                            void *stream)
{
    clear_error();
    if (!g || !y || P <= 0) {
        set_error("pff_relu_bwd: bad arguments");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_relu_bwd g", csg, offg, C));
    PFF_TRY(check_slice("pff_relu_bwd y", csy, offy, C));
    { k_relu_bwd<<<grid_for(P * C), 256, 0, S(stream)>>>(g, csg, offg, y, csy, offy, P, C); count_launch(); }
    return check_cuda("pff_relu_bwd");
}

extern "C" int pff_avgpool2(const bf16_t *x, int csx, int offx, bf16_t *y, int csy, int offy, int B, int H, int W,
                            int C, void *stream)
{
    clear_error();
    if (!x || !y || B <= 0 || H < 2 || W < 2 || H % 2 || W % 2) {
        set_error("pff_avgpool2: bad arguments (even H, W)");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_avgpool2 x", csx, offx, C));
    PFF_TRY(check_slice("pff_avgpool2 y", csy, offy, C));
    const long long n = (long long)B * (H / 2) * (W / 2) * C;
    { k_avgpool2<<<grid_for(n), 256, 0, S(stream)>>>(x, csx, offx, y, csy, offy, B, H, W, C); count_launch(); }
    return check_cuda("pff_avgpool2");
}

extern "C" int pff_avgpool2_bwd(const bf16_t *dy, int csd, int offd, bf16_t *dx, int csx, int offx, int B, int H,
                                int W, int C, int accumulate, void *stream)
{
    clear_error();
    if (!dy || !dx || B <= 0 || H < 2 || W < 2 || H % 2 || W % 2) {
        set_error("pff_avgpool2_bwd: bad arguments (even H, W)");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_avgpool2_bwd dy", csd, offd, C));
    PFF_TRY(check_slice("pff_avgpool2_bwd dx", csx, offx, C));
    const long long n = (long long)B * H * W * C;
    {
        k_avgpool2_bwd<<<grid_for(n), 256, 0, S(stream)>>>(dy, csd, offd, dx, csx, offx, B, H, W, C, accumulate);
        count_launch();
    }
    return check_cuda("pff_avgpool2_bwd");
}

extern "C" int pff_upsample2(const bf16_t *x, int csx, int offx, bf16_t *y, int csy, int offy, int B, int H, int W,
                             int C, void *stream)
{
    clear_error();
    if (!x || !y || B <= 0 || H <= 0 || W <= 0) {
        set_error("pff_upsample2: bad arguments");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_upsample2 x", csx, offx, C));
    PFF_TRY(check_slice("pff_upsample2 y", csy, offy, C));
    const long long n = (long long)B * 4 * H * W * C;
    { k_upsample2<<<grid_for(n), 256, 0, S(stream)>>>(x, csx, offx, y, csy, offy, B, H, W, C); count_launch(); }
    return check_cuda("pff_upsample2");
}

extern "C" int pff_upsample2_bwd(const bf16_t *dy, int csd, int offd, bf16_t *dx, int csx, int offx, int B, int H,
                                 int W, int C, void *stream)
{
    clear_error();
    if (!dy || !dx || B <= 0 || H <= 0 || W <= 0) {
        set_error("pff_upsample2_bwd: bad arguments");
        return PFF_ERR_ARG;
    }
    PFF_TRY(check_slice("pff_upsample2_bwd dy", csd, offd, C));
    PFF_TRY(check_slice("pff_upsample2_bwd dx", csx, offx, C));
    const long long n = (long long)B * H * W * C;
    { k_upsample2_bwd<<<grid_for(n), 256, 0, S(stream)>>>(dy, csd, offd, dx, csx, offx, B, H, W, C); count_launch(); }
    return check_cuda("pff_upsample2_bwd");
}

extern "C" int pff_mse_loss(const float *pred, int csp, const float *target, const float *weight, long long P,
                            bf16_t *dpred, int csd, float scale, float *loss, void *stream)
{
    clear_error();
    if (!pred || !target || !dpred || !loss || P <= 0 || csp <= 0 || csd <= 0) {
        set_error("pff_mse_loss: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_mse<<<grid_for(P), 256, 0, S(stream)>>>(pred, csp, target, weight, P, dpred, csd, scale, loss); count_launch(); }
    return check_cuda("pff_mse_loss");
}

extern "C" int pff_adam(float *p, const float *g, float *m, float *v, bf16_t *p_bf16, long long n, float lr, float b1,
                        float b2, float eps, int step, float weight_decay, void *stream)
{
    clear_error();
    if (!p || !g || !m || !v || n <= 0 || step < 1) {
        set_error("pff_adam: bad arguments");
        return PFF_ERR_ARG;
    }
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    {
        k_adam<<<grid_for(n), 256, 0, S(stream)>>>(p, g, m, v, p_bf16, n, lr, b1, b2, eps, bc1, bc2, weight_decay);
        count_launch();
    }
    return check_cuda("pff_adam");
}

extern "C" int pff_f32_to_bf16(const float *src, bf16_t *dst, long long n, void *stream)
{
    clear_error();
    if (!src || !dst || n <= 0) {
        set_error("pff_f32_to_bf16: bad arguments");
        return PFF_ERR_ARG;
    }
    { k_f32_to_bf16<<<grid_for(n), 256, 0, S(stream)>>>(src, dst, n); count_launch(); }
    return check_cuda("pff_f32_to_bf16");
}
