// libpff core: error plumbing, argument checks, and the D4 receiver stencil.
#include <cstdarg>
#include <cstring>
#include "pff_internal.h"

namespace pff {

static thread_local char g_err[512] = {0};
std::atomic<long long> g_launches{0};

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

int check_cuda(const char *where)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", where, cudaGetErrorString(e));
        return PFF_ERR_CUDA;
    }
    return PFF_OK;
}

int check_grid(int nx, int ny, int mode, const uint8_t *codes)
{
    if (nx < 2 || ny < 2) {
        set_error("grid must be at least 2x2 (got nx=%d, ny=%d)", nx, ny);
        return PFF_ERR_ARG;
    }
    if ((long long)nx * ny * 4LL >= (1LL << 31)) {
        set_error("grid too large for int32 donor indexing (nx*ny=%lld)", (long long)nx * ny);
        return PFF_ERR_ARG;
    }
    if (mode < 0 || mode > 3) {
        set_error("bound_mode must be 0..3 (got %d)", mode);
        return PFF_ERR_ARG;
    }
    if (mode == 3 && !codes) {
        set_error("custom bound_mode needs a device codes array");
        return PFF_ERR_ARG;
    }
    return PFF_OK;
}

// ---------------------------------------------------------------------------
// Receivers: pyfastflow/flow/receivers.py:31-58.
// One thread per cell of a 2-D block; the four neighbour loads of a block hit
// L1/L2 (each z row is read from DRAM once per block row band).
template <int MODE>
__global__ void __launch_bounds__(256) k_receivers(const float *__restrict__ z, int32_t *__restrict__ rcv,
                                                   float *__restrict__ grad, Grid g, float dx)
{
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y * blockDim.y + threadIdx.y;
    if (col >= g.nx || row >= g.ny) return;
    const int i = row * g.nx + col;
    const float zi = z[i];
    int r = i;
    float sr = 0.f;
    // A drop d can only beat the current best if d exceeds the best drop so far
    // (division by dx > 0 is monotone), so the IEEE division -- the costly part --
    // runs only for improving candidates; the comparison is still on the rounded
    // quotients, as in the reference (ties after rounding keep the earlier k).
    float dbest = 0.f;
    int js[4];
    neighbours4<MODE>(g, i, row, col, js);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int j = js[k];
        if (j != -1) {
            const float d = __fsub_rn(zi, __ldg(z + j));
            if (d > dbest) {
                const float tsr = __fdiv_rn(d, dx);
                if (tsr > sr) { sr = tsr; r = j; dbest = d; }
            }
        }
    }
    rcv[i] = r;
    grad[i] = sr;
}

template <int MODE>
static void launch_receivers(const float *z, int32_t *rcv, float *grad, const Grid &g, float dx,
                             cudaStream_t st)
{
    dim3 b(32, 8), gr(div_up(g.nx, 32), div_up(g.ny, 8));
    { k_receivers<MODE><<<gr, b, 0, st>>>(z, rcv, grad, g, dx); count_launch(); }
}

}  // namespace pff

using namespace pff;

extern "C" int pff_version(void) { return 100; }
extern "C" const char *pff_last_error_string(void) { return g_err; }
extern "C" long long pff_launch_count(void) { return g_launches.load(); }

extern "C" int pff_set_device(int device)
{
    clear_error();
    PFF_CUDA(cudaSetDevice(device));
    return PFF_OK;
}

extern "C" int pff_compute_receivers(const float *z, int32_t *receivers, float *gradient, int nx,
                                     int ny, float dx, int bound_mode, const uint8_t *codes,
                                     void *stream)
{
    clear_error();
    PFF_TRY(check_grid(nx, ny, bound_mode, codes));
    if (!z || !receivers || !gradient) {
        set_error("pff_compute_receivers: null pointer");
        return PFF_ERR_ARG;
    }
    Grid g{nx, ny, bound_mode, codes};
    PFF_MODE_DISPATCH(bound_mode, launch_receivers, z, receivers, gradient, g, dx, S(stream));
    return check_cuda("pff_compute_receivers");
}
