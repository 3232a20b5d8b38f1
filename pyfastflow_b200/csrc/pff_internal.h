// Host-side internals of libpff: status/error plumbing and workspace carving.
#pragma once
#include <cstddef>
#include <cstdint>
#include <atomic>
#include <cstdio>
#include <cuda_runtime.h>
#include "../../include/pff.h"
#include "pff_common.cuh"

namespace pff {

// Number of kernels this library has launched (all threads); read by benchmarks.
extern std::atomic<long long> g_launches;
inline void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// Timing probes (pff_probe_enable / pff_probe_read): PFF_PROBED(name, stream, launch)
// brackets `launch` with events on `stream` while probes are armed.
struct ProbeMark {
    int slot, idx;
};
ProbeMark probe_begin(const char *name, cudaStream_t st);
void probe_end(ProbeMark m, cudaStream_t st);
#define PFF_PROBED(name, st, ...)                                 \
    do {                                                          \
        const ::pff::ProbeMark _pm = ::pff::probe_begin(name, st); \
        __VA_ARGS__;                                              \
        ::pff::probe_end(_pm, st);                                \
    } while (0)

void set_error(const char *fmt, ...);
void clear_error();

// Internal status (never returned through the C ABI): a fast path that is not
// available here, so the caller takes its general path.
constexpr int PFF_ERR_UNSUPPORTED = 100;

// Returns PFF_ERR_CUDA (and records where) if the last launch/copy failed.
int check_cuda(const char *where);

#define PFF_TRY(expr)                         \
    do {                                      \
        int _rc = (expr);                     \
        if (_rc != PFF_OK) return _rc;        \
    } while (0)

#define PFF_CUDA(call)                                                     \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) {                                           \
            ::pff::set_error("%s: %s", #call, cudaGetErrorString(_e));    \
            return PFF_ERR_CUDA;                                           \
        }                                                                  \
    } while (0)

int check_grid(int nx, int ny, int mode, const uint8_t *codes);

// Read small device int arrays (a list of (pointer, count), at most 8 pointers and
// 64 ints) into host memory, in order, and synchronise `st`.  A one-thread kernel
// stores them into mapped pinned host memory, so the read uses no copy engine and
// does not wait behind bulk transfers other streams have in flight.
struct IntReads {
    const int *src[8];
    int n[8];
    int k = 0;
    IntReads &add(const int *p, int cnt)
    {
        src[k] = p;
        n[k++] = cnt;
        return *this;
    }
};
int read_ints(const IntReads &r, int *out, cudaStream_t st);


// Bump allocator over a caller-provided device workspace (256-byte aligned slices).
struct Carver {
    char *base;
    size_t cap, off;
    Carver(void *b, size_t c) : base((char *)b), cap(c), off(0) {}
    template <class T>
    T *take(size_t n)
    {
        size_t a = (off + 255) & ~size_t(255);
        off = a + n * sizeof(T);
        return (off <= cap && base) ? (T *)(base + a) : nullptr;
    }
    static size_t round(size_t n) { return (n + 255) & ~size_t(255); }
};

inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

// Launch helpers implemented per translation unit (declared for cross-TU use).
int launch_basin_init(int32_t *bid, const Grid &g, cudaStream_t st);
int run_labels(int32_t *bid, int32_t *rec_work, const Grid &g, int *round_flags, cudaStream_t st);
int count_pits(const int32_t *rec, const Grid &g, int *dev_count, int *pit_list, int *host_count,
               cudaStream_t st);

}  // namespace pff
