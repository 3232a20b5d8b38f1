// Shared device helpers for libpff: grid topology, packed keys, error plumbing.
//
// Grid topology restates pyfastflow/flow/neighbourer_flat.py:22-604 as runtime
// arguments (the reference bakes NX, NY, BOUND_MODE into each JIT'd kernel):
// row-major i = row*nx + col; direction k = 0 top, 1 left, 2 right, 3 bottom;
// boundary modes 0 normal, 1 periodic east-west, 2 periodic north-south,
// 3 custom u8 codes (0 nodata, 1 normal, 3 outlet, 7 inlet, 9 periodic).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pff {

__host__ __device__ __forceinline__ uint32_t f2u(float f)
{
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    __builtin_memcpy(&u, &f, 4);
    return u;
#endif
}
__host__ __device__ __forceinline__ float u2f(uint32_t u)
{
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    __builtin_memcpy(&f, &u, 4);
    return f;
#endif
}

struct Grid {
    int nx, ny;
    int mode;
    const uint8_t *codes;  // device pointer, custom mode only
    __host__ __device__ int N() const { return nx * ny; }
};

// which_edge (neighbourer_flat.py:75-110) from (row, col):
//   1 2 2 3 / 4 0 0 5 / 6 7 7 8
__device__ __forceinline__ int which_edge(int nx, int ny, int row, int col)
{
    if (row == 0) return col == 0 ? 1 : (col < nx - 1 ? 2 : 3);
    if (row < ny - 1) return col == 0 ? 4 : (col == nx - 1 ? 5 : 0);
    return col == 0 ? 6 : (col == nx - 1 ? 8 : 7);
}

// validate_link_n :146-159, validate_link_pew :228-237, validate_link_pns :305-314
__device__ __forceinline__ bool valid_n(int e, int k)
{
    if (e == 0) return true;
    if (k == 0) return e > 3;
    if (k == 1) return !(e == 1 || e == 4 || e == 6);
    if (k == 2) return !(e == 3 || e == 5 || e == 8);
    return e < 6;
}
__device__ __forceinline__ bool valid_pew(int e, int k)
{
    if (e == 0) return true;
    if (k == 0) return e > 3;
    if (k == 3) return e < 6;
    return true;
}
__device__ __forceinline__ bool valid_pns(int e, int k)
{
    if (e == 0) return true;
    if (k == 1) return !(e == 1 || e == 4 || e == 6);
    if (k == 2) return !(e == 3 || e == 5 || e == 8);
    return true;
}

// Raw neighbours: normal :124-141, periodic EW :194-223, periodic NS :271-300.
__device__ __forceinline__ int raw_n(int nx, int i, int k)
{
    return k == 0 ? i - nx : (k == 1 ? i - 1 : (k == 2 ? i + 1 : i + nx));
}
__device__ __forceinline__ int raw_pew(int nx, int i, int col, int k)
{
    if (k == 1) return col > 0 ? i - 1 : i + nx - 1;
    if (k == 2) return col < nx - 1 ? i + 1 : i - nx + 1;
    return raw_n(nx, i, k);
}
__device__ __forceinline__ int raw_pns(int nx, int ny, int i, int row, int k)
{
    if (k == 0) return row > 0 ? i - nx : i + nx * (ny - 1);
    if (k == 3) return row < ny - 1 ? i + nx : i - nx * (ny - 1);
    return raw_n(nx, i, k);
}

// neighbour (:542-569): index of the k-th neighbour of cell i = (row, col), or -1.
template <int MODE>
__device__ __forceinline__ int neighbour(const Grid &g, int i, int row, int col, int k)
{
    const int e = which_edge(g.nx, g.ny, row, col);
    if (MODE == 0) return valid_n(e, k) ? raw_n(g.nx, i, k) : -1;
    if (MODE == 1) return valid_pew(e, k) ? raw_pew(g.nx, i, col, k) : -1;
    if (MODE == 2) return valid_pns(e, k) ? raw_pns(g.nx, g.ny, i, row, k) : -1;
    // custom :360-462
    const int tb = g.codes[i];
    bool ok;
    if (tb == 0) ok = false;
    else if (tb != 9 || e == 0) ok = valid_n(e, k);
    else if (e <= 3 || e >= 6) ok = valid_pns(e, k);
    else ok = valid_pew(e, k);
    if (!ok) return -1;
    int node = (tb == 9) ? ((k == 0 || k == 3) ? raw_pns(g.nx, g.ny, i, row, k) : raw_pew(g.nx, i, col, k))
                         : raw_n(g.nx, i, k);
    if (node > -1 && node < g.N() && g.codes[node] == 0) node = -1;
    return node;
}

// can_leave_domain (:571-592)
template <int MODE>
__device__ __forceinline__ bool can_leave(const Grid &g, int i, int row, int col)
{
    if (MODE == 3) return g.codes[i] == 3;
    const int e = which_edge(g.nx, g.ny, row, col);
    if (MODE == 0) return e > 0;
    if (MODE == 1) return e != 0 && (e <= 3 || e >= 6);
    return e == 1 || e == 3 || e == 4 || e == 5 || e == 6 || e == 8;
}

// All four neighours of (row, col); interior cells of modes 0-2 (the bulk of
// any grid) skip the edge classification.
template <int MODE>
__device__ __forceinline__ void neighbours4(const Grid &g, int i, int row, int col, int (&j)[4])
{
    if (MODE != 3 && row > 0 && row < g.ny - 1 && col > 0 && col < g.nx - 1) {
        j[0] = i - g.nx; j[1] = i - 1; j[2] = i + 1; j[3] = i + g.nx;
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) j[k] = neighbour<MODE>(g, i, row, col, k);
}

template <int MODE>
__device__ __forceinline__ bool can_leave_i(const Grid &g, int i)
{
    if (MODE == 3) return g.codes[i] == 3;
    return can_leave<MODE>(g, i, i / g.nx, i % g.nx);
}
template <int MODE>
__device__ __forceinline__ int neighbour_i(const Grid &g, int i, int k)
{
    return neighbour<MODE>(g, i, i / g.nx, i % g.nx, k);
}

// Packed (f32, i32) key, f32_i32_struct.py:15-103: hi32 = raw bits for
// non-negative floats, (~bits) | 0x80000000 for negative ones; lo32 = index bits;
// compared as a signed 64-bit integer.
__host__ __device__ __forceinline__ long long pack_key(float f, int idx)
{
    const uint32_t u = f2u(f);
    const uint32_t hi = (u & 0x80000000u) ? ((~u) | 0x80000000u) : u;
    return (long long)(((unsigned long long)hi << 32) | (unsigned long long)(uint32_t)idx);
}
__host__ __device__ __forceinline__ int key_index(long long k) { return (int)(uint32_t)(unsigned long long)k; }
__host__ __device__ __forceinline__ float key_value(long long k)
{
    const uint32_t hi = (uint32_t)((unsigned long long)k >> 32);
    const uint32_t u = (hi & 0x80000000u) ? ((~hi) | 0x80000000u) : hi;
    return u2f(u);
}

// Candidate donors of j: the grid-adjacent cells and the wrap partners across
// opposite edges (every neighbour relation of every mode is among these).
__device__ __forceinline__ int donor_candidates(const Grid &g, int j, int row, int col, int *c)
{
    int n = 0;
    const int nx = g.nx, ny = g.ny;
    if (row > 0) c[n++] = j - nx;
    if (col > 0) c[n++] = j - 1;
    if (col < nx - 1) c[n++] = j + 1;
    if (row < ny - 1) c[n++] = j + nx;
    if (col == 0) c[n++] = j + nx - 1;
    if (col == nx - 1) c[n++] = j - nx + 1;
    if (row == 0) c[n++] = j + nx * (ny - 1);
    if (row == ny - 1) c[n++] = j - nx * (ny - 1);
    // ascending, without duplicates
    for (int a = 1; a < n; ++a) {
        int x = c[a], b = a - 1;
        while (b >= 0 && c[b] > x) { c[b + 1] = c[b]; --b; }
        c[b + 1] = x;
    }
    int m = 0;
    for (int a = 0; a < n; ++a)
        if (m == 0 || c[m - 1] != c[a]) c[m++] = c[a];
    return m;
}

// dispatch a templated launcher on the boundary mode
#define PFF_MODE_DISPATCH(mode, FN, ...)            \
    do {                                            \
        switch (mode) {                             \
        case 0: FN<0>(__VA_ARGS__); break;          \
        case 1: FN<1>(__VA_ARGS__); break;          \
        case 2: FN<2>(__VA_ARGS__); break;          \
        default: FN<3>(__VA_ARGS__); break;         \
        }                                           \
    } while (0)

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace pff
