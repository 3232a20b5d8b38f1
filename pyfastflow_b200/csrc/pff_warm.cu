// libpff warm-start glue: the GraphFlood warm-start network's input features and
// the map between its output (log depth) and an initial water depth.  No
// reference counterpart: the reference has no learned component.
//
// Inputs per cell (8 bf16 channels, NHWC rows):
//   0  elevation standardised per tile, (z - mean) / std
//   1  log local slope (steepest-descent gradient, floored at 1e-4), / 4 + 1
//   2  log drainage area in cells / log(cells per tile)
//   3  log(rainfall / 1e-5 m/s)
//   4  (Manning n - 0.04) / 0.02
//   5  log of the kinematic-wave depth (n P A / (dx sqrt(S)))^(3/5), + 1e-3, / 3
//   6, 7 zero
#include <cuda_bf16.h>
#include "pff_internal.h"

namespace pff {

typedef uint16_t bf16_t;

__device__ __forceinline__ bf16_t wf2bf(float f)
{
    __nv_bfloat16 b = __float2bfloat16_rn(f);
    return *reinterpret_cast<bf16_t *>(&b);
}

// mean and 1/std of each tile's elevation; one block per tile, double sums
__global__ void k_tile_stats(const float *__restrict__ z, long long N, float *stats)
{
    const float *zt = z + (long long)blockIdx.x * N;
    double s = 0.0, s2 = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = zt[i];
        s += v;
        s2 += v * v;
    }
    __shared__ double a[32], b[32];
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        a[threadIdx.x >> 5] = s;
        b[threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = 0.0, S2 = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            S += a[k];
            S2 += b[k];
        }
        const double m = S / N;
        const double var = fmax(S2 / N - m * m, 1e-12);
        stats[2 * blockIdx.x] = (float)m;
        stats[2 * blockIdx.x + 1] = (float)(1.0 / sqrt(var));
    }
}

__global__ void k_unet_features(const float *__restrict__ z, const float *__restrict__ slope,
                                const uint32_t *__restrict__ counts, const float *__restrict__ stats,
                                const float *__restrict__ prec, const float *__restrict__ manning, float dx,
                                long long N, int B, bf16_t *out)
{
    const float logN = logf((float)N);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)B * N;
         e += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(e / N);
        const float S = fmaxf(slope[e], 1e-4f);
        const float A = (float)counts[e];
        const float P = prec[t], n = manning[t];
        const float hk = powf(n * P * A * dx / sqrtf(S), 0.6f);  // A dx^2 / dx = A dx
        float f[8];
        f[0] = (z[e] - stats[2 * t]) * stats[2 * t + 1];
        f[1] = logf(S) * 0.25f + 1.f;
        f[2] = logf(A) / logN;
        f[3] = logf(P / 1e-5f);
        f[4] = (n - 0.04f) / 0.02f;
        f[5] = logf(hk + 1e-3f) / 3.f;
        f[6] = 0.f;
        f[7] = 0.f;
        uint4 pk;
        pk.x = (unsigned)wf2bf(f[0]) | ((unsigned)wf2bf(f[1]) << 16);
        pk.y = (unsigned)wf2bf(f[2]) | ((unsigned)wf2bf(f[3]) << 16);
        pk.z = (unsigned)wf2bf(f[4]) | ((unsigned)wf2bf(f[5]) << 16);
        pk.w = 0u;
        reinterpret_cast<uint4 *>(out)[e] = pk;
    }
}

// h0 = max(exp(min(pred, 5)) - eps, 0) from channel 0 of rows of cs floats; with a bed z, also
// the water surface zh = z + h0 (GraphFlood's state holds the surface, not the bed)
__global__ void k_unet_h0(const float *__restrict__ pred, int cs, float *h0, long long P, float eps,
                          const float *__restrict__ z, float *zh)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        // the log depth is capped at 5 (148 m): a prediction far outside the training
        // range must not reach the solver as an overflowing depth
        const float h = fmaxf(expf(fminf(pred[p * cs], 5.f)) - eps, 0.f);
        h0[p] = h;
        if (zh) zh[p] = __fadd_rn(z[p], h);
    }
}

// target = log(max(h, 0) + eps); a NaN depth counts as dry
__global__ void k_unet_target(const float *__restrict__ h, float *tgt, long long P, float eps)
{
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
        const float v = h[p];
        tgt[p] = logf((v > 0.f ? v : 0.f) + eps);
    }
}

}  // namespace pff

using namespace pff;

extern "C" int pff_unet_features(const float *z, const float *slope, const uint32_t *counts, const float *prec,
                                 const float *manning, float dx, int B, long long N, float *stats, bf16_t *out,
                                 void *stream)
{
    clear_error();
    if (!z || !slope || !counts || !prec || !manning || !stats || !out || B <= 0 || N <= 1 || !(dx > 0.f)) {
        set_error("pff_unet_features: bad arguments");
        return PFF_ERR_ARG;
    }
    cudaStream_t st = S(stream);
    { k_tile_stats<<<B, 256, 0, st>>>(z, N, stats); count_launch(); }
    const long long n = (long long)B * N;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    { k_unet_features<<<blocks, 256, 0, st>>>(z, slope, counts, stats, prec, manning, dx, N, B, out); count_launch(); }
    return check_cuda("pff_unet_features");
}

extern "C" int pff_unet_h0(const float *pred, int cs, float *h0, long long P, float eps, const float *z, float *zh,
                           void *stream)
{
    clear_error();
    if (!pred || !h0 || P <= 0 || cs <= 0 || (zh && !z)) {
        set_error("pff_unet_h0: bad arguments");
        return PFF_ERR_ARG;
    }
    const int blocks = (int)std::min<long long>((P + 255) / 256, 148LL * 16);
    { k_unet_h0<<<blocks, 256, 0, S(stream)>>>(pred, cs, h0, P, eps, z, zh); count_launch(); }
    return check_cuda("pff_unet_h0");
}

extern "C" int pff_unet_target(const float *h, float *target, long long P, float eps, void *stream)
{
    clear_error();
    if (!h || !target || P <= 0) {
        set_error("pff_unet_target: bad arguments");
        return PFF_ERR_ARG;
    }
    const int blocks = (int)std::min<long long>((P + 255) / 256, 148LL * 16);
    { k_unet_target<<<blocks, 256, 0, S(stream)>>>(h, target, P, eps); count_launch(); }
    return check_cuda("pff_unet_target");
}
