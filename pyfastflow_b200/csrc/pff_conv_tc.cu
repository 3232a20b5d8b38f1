// libpff 3x3 convolution on the 5th-generation tensor cores (tcgen05): the
// forward / data-gradient GEMM of the warm-start U-Net when Cin and Cout are
// multiples of 64.  No reference counterpart (the reference has no network).
//
// Implicit GEMM, M = 128 pixels (a BH x BW block of one image, BH * BW = 128),
// N = 64 or 128 output channels, K = 9 taps x Cin.  Per K step (one tap, 64 input
// channels):
//   - TMA loads the A box (64 channels x BW x BH pixels of image b, shifted by the
//     tap) straight from the NHWC activations; out-of-image rows and columns are
//     zero-filled by the TMA unit, which is the convolution's padding.  The box
//     lands as 128 rows of 128 bytes with the 128-byte swizzle: the canonical
//     K-major operand layout of tcgen05.mma.
//   - TMA loads the B box (64 K values x N output channels) of the [Cout][9*Cin]
//     weights the same way.
//   - one thread issues 4 tcgen05.mma (K = 16 each) accumulating in TMEM.
// A 4-stage mbarrier pipeline overlaps loads and MMAs: one thread produces (TMA),
// one issues MMAs and commits each stage back to the producer; after the last
// commit the 4 warps read the 128 x N accumulator with tcgen05.ld (warp w owns
// TMEM lanes 32w..32w+31 = pixels), add the bias, apply ReLU and store bf16 or f32.
// Every mbarrier wait is bounded; a wait that runs out sets an error flag.  The
// block then waits (again bounded) for every TMA load it issued but did not
// consume, so that no bulk copy is still writing its shared memory when it frees
// its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include "pff_internal.h"

namespace pff {

typedef uint16_t bf16_t;

constexpr int TC_BM = 128, TC_BK = 64, TC_ST = 4, TC_THREADS = 128;
constexpr unsigned long long TC_WAIT_NS = 1000000000ull;  // a wait gives up after 1 s

__device__ __forceinline__ unsigned tc_smem(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *b, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(tc_smem(b)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc_smem(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// bounded wait for the phase with parity `ph` to complete; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t *b, unsigned ph)
{
    const unsigned a = tc_smem(b);
    const unsigned long long t0 = gtimer();
    for (;;) {
        unsigned done;
        asm volatile(
            "{\n.reg .pred p;\n"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.b32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(ph)
            : "memory");
        if (done) return true;
        if (gtimer() - t0 > TC_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1, int c2,
                                            int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
        "[%2];\n" ::"r"(tc_smem(dst)),
        "l"(map), "r"(tc_smem(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];\n" ::"r"(
            tc_smem(dst)),
        "l"(map), "r"(tc_smem(bar)), "r"(c0), "r"(c1)
        : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t umma_desc(unsigned saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                          // leading byte offset (unused with this swizzle)
    d |= (uint64_t)(1024 >> 4) << 32;                // stride byte offset
    d |= (uint64_t)1 << 46;                          // descriptor version
    d |= (uint64_t)2 << 61;                          // 128-byte swizzle
    return d;
}

// instruction descriptor: D f32, A and B bf16, both K-major, M x N
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_f16(unsigned tmem_d, uint64_t da, uint64_t db, uint32_t idesc, unsigned acc)
{
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(tc_smem(bar))
                 : "memory");
}

struct TcArgs {
    const float *bias;
    void *y;
    int csy, offy;
    int B, H, W, Cin, Cout;
    int BW, BH;  // pixel block, BW * BH = 128
    int relu, out_f32;
    int offx;    // channel offset of the input slice (first TMA coordinate)
    int *err;
};

template <int BN>
__global__ void __launch_bounds__(TC_THREADS) k_conv3x3_tc(const __grid_constant__ CUtensorMap mapA,
                                                           const __grid_constant__ CUtensorMap mapB, TcArgs a)
{
    extern __shared__ uint8_t dsmem[];
    // stages 1024-byte aligned (the 128-byte swizzle repeats every 8 rows of 128 B)
    uint8_t *base = (uint8_t *)(((uintptr_t)dsmem + 1023) & ~(uintptr_t)1023);
    constexpr int ABYTES = TC_BM * TC_BK * 2, BBYTES = BN * TC_BK * 2;
    uint8_t *sA = base;
    uint8_t *sB = base + TC_ST * ABYTES;
    __shared__ __align__(8) uint64_t full[TC_ST], empty[TC_ST], done;
    __shared__ unsigned tmem_base;
    __shared__ int failed;
    __shared__ int issued, consumed;  // TMA stages issued by the producer / waited for by the MMA issuer
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    const int tiles_x = a.W / a.BW, tiles_y = a.H / a.BH;
    int t = blockIdx.x;
    const int bx = t % tiles_x;
    t /= tiles_x;
    const int by = t % tiles_y;
    const int b = t / tiles_y;
    const int x0 = bx * a.BW, y0 = by * a.BH;
    const int n0 = blockIdx.y * BN;
    const int kchunks = a.Cin / TC_BK;
    const int nk = 9 * kchunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_ST; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        failed = 0;
        issued = 0;
        consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {  // TMEM: BN f32 columns x 128 lanes
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc_smem(&tmem_base)),
                     "r"((unsigned)BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const unsigned tmem = tmem_base;

    if (warp == 0 && lane == 0) {  // producer
        int n = 0;
        for (int it = 0; it < nk; ++it) {
            const int s = it % TC_ST;
            if (it >= TC_ST && !mbar_wait(&empty[s], ((it / TC_ST) - 1) & 1)) { failed = 1; break; }
            if (*(volatile int *)&failed) break;  // the MMA issuer gave up: issue nothing more
            const int tap = it / kchunks, kc = it - tap * kchunks;
            const int dy = tap / 3 - 1, dx = tap % 3 - 1;
            mbar_expect_tx(&full[s], ABYTES + BBYTES);
            tma_load_4d(sA + s * ABYTES, &mapA, &full[s], a.offx + kc * TC_BK, x0 + dx, y0 + dy, b);
            tma_load_2d(sB + s * BBYTES, &mapB, &full[s], tap * a.Cin + kc * TC_BK, n0);
            n = it + 1;
        }
        issued = n;
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        constexpr uint32_t idesc = umma_idesc(TC_BM, BN);
        bool ok = true;
        int n = 0;
        for (int it = 0; it < nk; ++it) {
            const int s = it % TC_ST;
            if (!mbar_wait(&full[s], (it / TC_ST) & 1)) { ok = false; break; }
            n = it + 1;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const unsigned abase = tc_smem(sA + s * ABYTES), bbase = tc_smem(sB + s * BBYTES);
#pragma unroll
            for (int k = 0; k < TC_BK / 16; ++k)  // K = 16 per MMA: +32 bytes within the swizzled rows
                umma_f16(tmem, umma_desc(abase + 32 * k), umma_desc(bbase + 32 * k), idesc, (it | k) ? 1u : 0u);
            umma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        consumed = n;
        if (!ok) failed = 1;
        umma_commit(&done);  // arrives when every MMA issued so far has completed
    }
    __syncwarp();
    // epilogue: every warp reads its 32 TMEM lanes (pixels)
    const bool ready = mbar_wait(&done, 0);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (!ready) failed = 1;
    __syncthreads();
    if (failed && threadIdx.x == 0) {
        // Loads issued but never consumed may still be landing in this block's
        // shared memory: wait for each (at most one per stage, since the producer
        // waits for a stage to be freed before it reloads it).
        for (int it = consumed; it < issued; ++it) mbar_wait(&full[it % TC_ST], (it / TC_ST) & 1);
    }
    __syncthreads();
    const bool good = !failed;
    const int r = warp * 32 + lane;  // accumulator row = pixel of the block
    const int py = y0 + r / a.BW, px = x0 + r % a.BW;
    const long long p = ((long long)b * a.H + py) * a.W + px;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
        unsigned v[16];
        const unsigned taddr = tmem + ((unsigned)(warp * 32) << 16) + (unsigned)c;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (!good) continue;
        float f[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int co = n0 + c + q;
            float x = __uint_as_float(v[q]);
            if (a.bias) x += a.bias[co];
            if (a.relu) x = fmaxf(x, 0.f);
            f[q] = x;
        }
        if (a.out_f32) {
            float4 *yo = reinterpret_cast<float4 *>((float *)a.y + p * a.csy + a.offy + n0 + c);
#pragma unroll
            for (int q = 0; q < 4; ++q) yo[q] = make_float4(f[4 * q], f[4 * q + 1], f[4 * q + 2], f[4 * q + 3]);
        } else {
            uint4 *yo = reinterpret_cast<uint4 *>((bf16_t *)a.y + p * a.csy + a.offy + n0 + c);
            unsigned w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                __nv_bfloat162 h2 = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
                w[q] = *reinterpret_cast<unsigned *>(&h2);
            }
            yo[0] = make_uint4(w[0], w[1], w[2], w[3]);
            yo[1] = make_uint4(w[4], w[5], w[6], w[7]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"((unsigned)BN));
    }
    if (threadIdx.x == 0 && failed) atomicOr(a.err, 1);
}

// ---- host side ------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

static int g_conv_path = 0;  // 0 automatic (default), 1 mma.sync only, 2 tcgen05 only
static int *g_tc_err[64] = {nullptr};

// Whether the tcgen05 kernel applies: channel counts, slice offsets and a pixel block
bool conv_tc_supported(int H, int W, int Cin, int Cout, int csx, int offx, int csy, int offy, int out_f32, int *BW,
                       int *BH)
{
    if (Cin % TC_BK || Cout % 64 || offx % TC_BK || csx % 8 || csy % 8 || offy % 8) return false;
    if (out_f32 && (csy % 4 || offy % 4)) return false;
    const int bw = W >= 128 ? 128 : W;
    if (bw <= 0 || 128 % bw || W % bw) return false;
    const int bh = 128 / bw;
    if (H % bh) return false;
    *BW = bw;
    *BH = bh;
    return true;
}

int conv3x3_tc(const bf16_t *x, int csx, int offx, const bf16_t *w, const float *bias, void *y, int csy, int offy,
               int B, int H, int W, int Cin, int Cout, int relu, int out_f32, cudaStream_t st)
{
    int BW = 0, BH = 0;
    if (!conv_tc_supported(H, W, Cin, Cout, csx, offx, csy, offy, out_f32, &BW, &BH)) {
        set_error("pff_conv3x3_fwd: shape not supported by the tcgen05 path");
        return PFF_ERR_ARG;
    }
    EncodeTiledFn enc = encode_fn();
    if (!enc) {
        set_error("pff_conv3x3_fwd: cuTensorMapEncodeTiled unavailable");
        return PFF_ERR_CUDA;
    }
    CUtensorMap mA, mB;
    {
        const cuuint64_t dims[4] = {(cuuint64_t)csx, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
        const cuuint64_t strides[3] = {(cuuint64_t)csx * 2, (cuuint64_t)W * csx * 2, (cuuint64_t)H * W * csx * 2};
        const cuuint32_t box[4] = {(cuuint32_t)TC_BK, (cuuint32_t)BW, (cuuint32_t)BH, 1};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        CUresult r = enc(&mA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)x, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("pff_conv3x3_fwd: activation tensor map (error %d)", (int)r);
            return PFF_ERR_ARG;
        }
    }
    const int BN = (Cout % 128 == 0) ? 128 : 64;
    {
        const cuuint64_t dims[2] = {(cuuint64_t)(9 * Cin), (cuuint64_t)Cout};
        const cuuint64_t strides[1] = {(cuuint64_t)9 * Cin * 2};
        const cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)BN};
        const cuuint32_t es[2] = {1, 1};
        CUresult r = enc(&mB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)w, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("pff_conv3x3_fwd: weight tensor map (error %d)", (int)r);
            return PFF_ERR_ARG;
        }
    }
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("pff_conv3x3_fwd: device %d out of range", dev);
        return PFF_ERR_ARG;
    }
    if (!g_tc_err[dev]) {
        PFF_CUDA(cudaMalloc(&g_tc_err[dev], sizeof(int)));
        PFF_CUDA(cudaMemset(g_tc_err[dev], 0, sizeof(int)));
    }
    TcArgs args{bias, y, csy, offy, B, H, W, Cin, Cout, BW, BH, relu, out_f32, offx, g_tc_err[dev]};
    const size_t smem = (size_t)TC_ST * (TC_BM * TC_BK * 2 + BN * TC_BK * 2) + 1024;
    dim3 grid((unsigned)(B * (H / BH) * (W / BW)), (unsigned)(Cout / BN));
    if (BN == 128) {
        PFF_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        { k_conv3x3_tc<128><<<grid, TC_THREADS, smem, st>>>(mA, mB, args); count_launch(); }
    } else {
        PFF_CUDA(cudaFuncSetAttribute(k_conv3x3_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        { k_conv3x3_tc<64><<<grid, TC_THREADS, smem, st>>>(mA, mB, args); count_launch(); }
    }
    return check_cuda("pff_conv3x3_fwd (tcgen05)");
}

}  // namespace pff

using namespace pff;

extern "C" int pff_conv_set_path(int path)
{
    clear_error();
    if (path < 0 || path > 2) {
        set_error("pff_conv_set_path: 0 automatic, 1 mma.sync, 2 tcgen05");
        return PFF_ERR_ARG;
    }
    g_conv_path = path;
    return PFF_OK;
}

extern "C" int pff_conv_tc_status(int *flag)
{
    clear_error();
    if (!flag) {
        set_error("pff_conv_tc_status: null pointer");
        return PFF_ERR_ARG;
    }
    int dev = 0;
    PFF_CUDA(cudaGetDevice(&dev));
    *flag = 0;
    if (dev >= 0 && dev < 64 && g_tc_err[dev]) {
        PFF_CUDA(cudaMemcpy(flag, g_tc_err[dev], sizeof(int), cudaMemcpyDeviceToHost));
        PFF_CUDA(cudaMemset(g_tc_err[dev], 0, sizeof(int)));
    }
    return PFF_OK;
}

namespace pff {
int conv_path() { return g_conv_path; }
}
