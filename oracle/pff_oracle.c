/*
 * pff_oracle — CPU restatement of pyfastflow's flow-routing / graphflood hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and by
 * bench.py's CPU-baseline / reference legs as the checker and the timed CPU
 * implementation of the reference algorithm.  The product library (libpff.so)
 * never links, loads or calls it.
 *
 * The reference (bgailleton/pyfastflow, Python on the Taichi DSL) cannot run in
 * this environment (no taichi).  Parity is pinned by
 *   - the reference's own key-format checks (archive/test_pack_unpack.py:16-26,
 *     :68-77, :175-230) for pack/unpack,
 *   - hand-derived known-answer grids and independent cross-checks (drainage
 *     counts == topological-order accumulation) for everything else,
 * because the reference ships no golden vectors for receivers, labels, reroute,
 * accumulation or graphflood.
 *
 * Semantics: serial ascending-index execution of each top-level Taichi loop
 * (what Taichi's CPU backend does with one thread).  With nthreads > 1 the
 * race-free loops run under OpenMP (used only to time the CPU baseline).
 *
 * Grid topology restates flow/neighbourer_flat.py:22-604 (row-major i = row*nx +
 * col; direction k = 0 top, 1 left, 2 right, 3 bottom; boundary modes 0 normal,
 * 1 periodic east-west, 2 periodic north-south, 3 custom u8 codes 0/1/3/7/9).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

typedef struct {
    int nx, ny;
    int mode;               /* 0 normal, 1 periodic EW, 2 periodic NS, 3 custom */
    const uint8_t *codes;   /* N custom codes, mode 3 only */
} orc_grid;

int orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

int orc_ceil_log2(long long n)
{
    /* math.ceil(math.log2(n)) for n >= 1 */
    int r = 0;
    long long p = 1;
    while (p < n) { p <<= 1; ++r; }
    return r;
}

/* ---- neighbourer_flat.py -------------------------------------------------- */

/* which_edge :75-110 — 0 interior, 1..8 = corners/edges, layout
 *   1 2 2 3 / 4 0 0 5 / 6 7 7 8                                                */
static inline int which_edge(const orc_grid *g, int i)
{
    const int nx = g->nx, ny = g->ny, N = nx * ny;
    const int tx = i % nx, ty = i / nx;
    if (i == 0) return 1;
    if (i < nx - 1) return 2;
    if (i == nx - 1) return 3;
    if (i < N - nx) return tx == 0 ? 4 : (tx == nx - 1 ? 5 : 0);
    if (ty == ny - 1) return tx == 0 ? 6 : (tx == nx - 1 ? 8 : 7);
    return 0;
}

/* validate_link_n :146-159 */
static inline int valid_n(int e, int k)
{
    if (e == 0) return 1;
    if (k == 0) return !(e <= 3);
    if (k == 1) return !(e == 1 || e == 4 || e == 6);
    if (k == 2) return !(e == 3 || e == 5 || e == 8);
    return !(e >= 6);
}
/* validate_link_pew :228-237 */
static inline int valid_pew(int e, int k)
{
    if (e == 0) return 1;
    if (k == 0) return !(e <= 3);
    if (k == 3) return !(e >= 6);
    return 1;
}
/* validate_link_pns :305-314 */
static inline int valid_pns(int e, int k)
{
    if (e == 0) return 1;
    if (k == 1) return !(e == 1 || e == 4 || e == 6);
    if (k == 2) return !(e == 3 || e == 5 || e == 8);
    return 1;
}
/* raw neighbours: normal :124-141, periodic EW :194-223, periodic NS :271-300 */
static inline int raw_n(const orc_grid *g, int i, int k)
{
    switch (k) { case 0: return i - g->nx; case 1: return i - 1; case 2: return i + 1; default: return i + g->nx; }
}
static inline int raw_pew(const orc_grid *g, int i, int k)
{
    const int nx = g->nx, col = i % nx;
    switch (k) {
    case 0: return i - nx;
    case 1: return col > 0 ? i - 1 : i + nx - 1;
    case 2: return col < nx - 1 ? i + 1 : i - nx + 1;
    default: return i + nx;
    }
}
static inline int raw_pns(const orc_grid *g, int i, int k)
{
    const int nx = g->nx, ny = g->ny, row = i / nx;
    switch (k) {
    case 0: return row > 0 ? i - nx : i + nx * (ny - 1);
    case 1: return i - 1;
    case 2: return i + 1;
    default: return row < ny - 1 ? i + nx : i - nx * (ny - 1);
    }
}
/* custom codes :360-462 */
static inline int nb_custom(const orc_grid *g, int i, int k)
{
    const int N = g->nx * g->ny;
    const int tb = g->codes[i];
    const int e = which_edge(g, i);
    int ok;
    if (tb == 0) ok = 0;
    else if (tb != 9) ok = valid_n(e, k);
    else if (e == 0) ok = valid_n(e, k);
    else if (e <= 3 || e >= 6) ok = valid_pns(e, k);
    else ok = valid_pew(e, k);
    if (!ok) return -1;
    int node;
    if (tb == 9) node = (k == 0 || k == 3) ? raw_pns(g, i, k) : raw_pew(g, i, k);
    else node = raw_n(g, i, k);
    if (node > -1 && node < N && g->codes[node] == 0) node = -1;
    return node;
}

/* neighbour :542-569 */
int orc_neighbour(const orc_grid *g, int i, int k)
{
    switch (g->mode) {
    case 0: return valid_n(which_edge(g, i), k) ? raw_n(g, i, k) : -1;
    case 1: return valid_pew(which_edge(g, i), k) ? raw_pew(g, i, k) : -1;
    case 2: return valid_pns(which_edge(g, i), k) ? raw_pns(g, i, k) : -1;
    default: return nb_custom(g, i, k);
    }
}

/* can_leave_domain :571-592 (normal :183, pew :259, pns :337, custom :465) */
int orc_can_leave(const orc_grid *g, int i)
{
    const int e = which_edge(g, i);
    switch (g->mode) {
    case 0: return e > 0;
    case 1: return (e <= 3 || e >= 6) && e != 0;
    case 2: return e == 1 || e == 3 || e == 4 || e == 5 || e == 6 || e == 8;
    default: return g->codes[i] == 3;
    }
}

void orc_neighbour_table(const orc_grid *g, int32_t *nbr4, uint8_t *leave)
{
    const int N = g->nx * g->ny;
    for (int i = 0; i < N; ++i) {
        for (int k = 0; k < 4; ++k) nbr4[4 * i + k] = orc_neighbour(g, i, k);
        leave[i] = (uint8_t)orc_can_leave(g, i);
    }
}

/* ---- f32_i32_struct.py:15-103 — packed (f32, i32) lexicographic key ------- */
int64_t orc_pack_float_index(float f, int32_t idx)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    /* flip_float_bits :15-30 then upper-half complement :67-73 */
    uint32_t fenc = (u & 0x80000000u) ? (u ^ 0x80000000u) : ~u;
    uint64_t packed = ((uint64_t)fenc << 32) | (uint64_t)(uint32_t)idx;
    uint64_t up = (~packed) & 0xFFFFFFFF00000000ull;
    uint64_t lo = packed & 0xFFFFFFFFull;
    return (int64_t)(up | lo);
}
void orc_unpack_float_index(int64_t key, float *f, int32_t *idx)
{
    uint64_t p = (uint64_t)key;
    uint64_t up = (~p) & 0xFFFFFFFF00000000ull;
    uint64_t un = up | (p & 0xFFFFFFFFull);
    uint32_t fenc = (uint32_t)(un >> 32);
    uint32_t ienc = (uint32_t)(un & 0xFFFFFFFFull);
    uint32_t r = (fenc & 0x80000000u) ? ~fenc : (fenc ^ 0x80000000u); /* unflip :33-48 */
    memcpy(f, &r, 4);
    *idx = (int32_t)ienc;
}

/* Same ordering for doubles (FP64 run only): (ordered bits, unsigned index). */
typedef struct { int64_t hi; uint32_t lo; } orc_key64;
static inline orc_key64 key64_make(double d, int32_t idx)
{
    uint64_t b;
    memcpy(&b, &d, 8);
    orc_key64 k;
    k.hi = (b >> 63) ? (int64_t)((~b) | 0x8000000000000000ull) : (int64_t)b;
    k.lo = (uint32_t)idx;
    return k;
}
static inline void key64_split(orc_key64 k, double *d, int32_t *idx)
{
    uint64_t h = (uint64_t)k.hi;
    uint64_t b = (h >> 63) ? ((~h) | 0x8000000000000000ull) : h;
    memcpy(d, &b, 8);
    *idx = (int32_t)k.lo;
}
static inline int key64_less(orc_key64 a, orc_key64 b)
{
    return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}
static inline int key64_eq(orc_key64 a, orc_key64 b) { return a.hi == b.hi && a.lo == b.lo; }

static inline void key32_split(int64_t k, float *f, int *idx) { orc_unpack_float_index(k, f, idx); }

/* ---- lakeflow.py integer kernels ----------------------------------------- */

/* depression_counter :25-44 */
int orc_depression_counter(const int32_t *rec, const orc_grid *g)
{
    const int N = g->nx * g->ny;
    int n = 0;
    for (int i = 0; i < N; ++i)
        if (rec[i] == i && !orc_can_leave(g, i)) ++n;
    return n;
}
/* basin_id_init :47-61 */
void orc_basin_id_init(int32_t *bid, const orc_grid *g)
{
    const int N = g->nx * g->ny;
    for (int i = 0; i < N; ++i) bid[i] = orc_can_leave(g, i) ? 0 : i + 1;
}
/* propagate_basin :64-80 (serial, in place) */
void orc_propagate_basin(int32_t *bid, int32_t *rec_, int N)
{
    for (int i = 0; i < N; ++i) {
        bid[i] = bid[rec_[i]];
        rec_[i] = rec_[rec_[i]];
    }
}
/* basin_identification :82-101 — labels of the receiver forest `rec`. */
void orc_basin_identification(int32_t *bid, const int32_t *rec, int32_t *rec_, const orc_grid *g)
{
    const int N = g->nx * g->ny;
    memcpy(rec_, rec, sizeof(int32_t) * (size_t)N);
    orc_basin_id_init(bid, g);
    const int n = orc_ceil_log2(N) + 1;
    for (int r = 0; r < n; ++r) orc_propagate_basin(bid, rec_, N);
}

/* ---- downstream_propag.py — rake and compress ----------------------------- */

/* getSrc :21-39 */
static inline int get_src(const int32_t *src, int t, int it)
{
    int e = src[t];
    int flip = e < 0;
    if ((e < 0 ? -e : e) == it + 1) flip = !flip;
    return flip;
}
/* rcv2donor :78-96 (serial: donor slots fill in ascending donor index) */
void orc_rcv2donor(const int32_t *rcv, int32_t *dnr, int32_t *ndnr, int N)
{
    for (int t = 0; t < N; ++t) {
        if (rcv[t] == t) continue;
        int old = ndnr[rcv[t]]++;
        long long did = (long long)rcv[t] * 4 + old;
        if (did < (long long)N * 4) dnr[did] = t;
    }
}

#define RC_BODY(PT)                                                                 \
    for (int tid = 0; tid < N; ++tid) {                                             \
        const int flip = get_src(src, tid, it);                                     \
        int worked = 0;                                                             \
        int donors[4] = {-1, -1, -1, -1};                                           \
        int todo = flip ? ndnr_[tid] : ndnr[tid];                                   \
        const long long base = (long long)tid * 4;                                  \
        PT padd = 0;                                                                \
        int i = 0;                                                                  \
        while (i < todo && i < 4) {                                                 \
            if (donors[i] == -1) donors[i] = flip ? dnr_[base + i] : dnr[base + i]; \
            const int did = donors[i];                                              \
            const int fd = get_src(src, did, it);                                   \
            const int nd = fd ? ndnr_[did] : ndnr[did];                             \
            if (nd <= 1) {                                                          \
                if (!worked) padd = flip ? p_[tid] : p[tid];                        \
                worked = 1;                                                         \
                padd += fd ? p_[did] : p[did];                                      \
                if (nd == 0) {                                                      \
                    --todo;                                                         \
                    if (todo > i && base + todo < (long long)N * 4)                 \
                        donors[i] = flip ? dnr_[base + todo] : dnr[base + todo];    \
                    --i;                                                            \
                } else {                                                            \
                    donors[i] = fd ? dnr_[(long long)did * 4] : dnr[(long long)did * 4]; \
                }                                                                   \
            }                                                                       \
            ++i;                                                                    \
        }                                                                           \
        if (worked) {                                                               \
            const int m = todo < 4 ? todo : 4;                                      \
            if (flip) {                                                             \
                ndnr[tid] = todo; p[tid] = padd;                                    \
                for (int j = 0; j < m; ++j) dnr[base + j] = donors[j];              \
            } else {                                                                \
                ndnr_[tid] = todo; p_[tid] = padd;                                  \
                for (int j = 0; j < m; ++j) dnr_[base + j] = donors[j];             \
            }                                                                       \
            src[tid] = (flip ? 1 : -1) * (it + 1);  /* updateSrc :43-56 */          \
        }                                                                           \
    }

/* rake_compress_accum :100-179, one round, f32 payload (reference) */
int orc_rake_compress_accum(int32_t *dnr, int32_t *ndnr, float *p, int32_t *src,
                            int32_t *dnr_, int32_t *ndnr_, float *p_, int it, int N)
{
    RC_BODY(float)
    return 0;
}
/* same round with an integer payload (exact drainage counts) */
int orc_rake_compress_accum_u32(int32_t *dnr, int32_t *ndnr, uint32_t *p, int32_t *src,
                                int32_t *dnr_, int32_t *ndnr_, uint32_t *p_, int it, int N)
{
    RC_BODY(uint32_t)
    return 0;
}
/* fuse :60-74 */
void orc_fuse(float *A, const int32_t *src, const float *B, int it, int N)
{
    for (int t = 0; t < N; ++t) if (get_src(src, t, it)) A[t] = B[t];
}
void orc_fuse_u32(uint32_t *A, const int32_t *src, const uint32_t *B, int it, int N)
{
    for (int t = 0; t < N; ++t) if (get_src(src, t, it)) A[t] = B[t];
}

/* Whole accumulation as FlowRouter.accumulate_constant_Q drives it
 * (flow/flowfields.py:272-292): Q holds the per-cell seed on entry (the
 * reference's Q.fill), the upstream sum on exit.  Returns the number of rounds
 * that did work (diagnostic).  ws: int32 workspace of 10*N. */
int orc_accumulate(const int32_t *rcv, float *Q, uint32_t *cnt, int N, int32_t *ws,
                   int32_t *active_per_round)
{
    int32_t *dnr = ws, *dnr_ = ws + 4 * (size_t)N, *ndnr = ws + 8 * (size_t)N,
            *ndnr_ = ws + 9 * (size_t)N;
    /* every buffer starts zeroed, as Taichi fields do */
    int32_t *src = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    float *Q_ = (float *)calloc((size_t)N, sizeof(float));
    uint32_t *c_ = (uint32_t *)calloc((size_t)N, sizeof(uint32_t));
    int32_t *ndnr_c = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    int32_t *ndnrc_ = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    int32_t *dnr_c = (int32_t *)calloc(4 * (size_t)N, sizeof(int32_t));
    int32_t *dnrc_ = (int32_t *)calloc(4 * (size_t)N, sizeof(int32_t));
    int32_t *src_c = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    const int logn = orc_ceil_log2(N) + 1;
    memset(ws, 0, sizeof(int32_t) * 10 * (size_t)N);
    orc_rcv2donor(rcv, dnr, ndnr, N);
    if (cnt) {
        memcpy(ndnr_c, ndnr, sizeof(int32_t) * (size_t)N);
        memcpy(dnr_c, dnr, sizeof(int32_t) * 4 * (size_t)N);
        memset(src_c, 0, sizeof(int32_t) * (size_t)N);
        for (int i = 0; i < N; ++i) cnt[i] = 1;
    }
    int worked_rounds = 0;
    for (int it = 0; it <= logn; ++it) {
        if (active_per_round) {
            int a = 0;
            for (int t = 0; t < N; ++t) {
                int f = get_src(src, t, it);
                if ((f ? ndnr_[t] : ndnr[t]) > 0) ++a;
            }
            active_per_round[it] = a;
            if (a) worked_rounds = it + 1;
        }
        orc_rake_compress_accum(dnr, ndnr, Q, src, dnr_, ndnr_, Q_, it, N);
        if (cnt) orc_rake_compress_accum_u32(dnr_c, ndnr_c, cnt, src_c, dnrc_, ndnrc_, c_, it, N);
    }
    orc_fuse(Q, src, Q_, logn, N);
    if (cnt) orc_fuse_u32(cnt, src_c, c_, logn, N);
    free(src); free(Q_); free(c_); free(ndnr_c); free(ndnrc_); free(dnr_c); free(dnrc_); free(src_c);
    return worked_rounds;
}

/* Independent cross-check: exact accumulation in topological order (Kahn) of
 * any receiver forest; returns -1 if the receivers contain a cycle. */
int orc_topo_accumulate_u32(const int32_t *rcv, uint32_t *cnt, int N)
{
    int32_t *indeg = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N; ++i) { cnt[i] = 1; if (rcv[i] != i) indeg[rcv[i]]++; }
    int h = 0, t = 0;
    for (int i = 0; i < N; ++i) if (indeg[i] == 0) q[t++] = i;
    while (h < t) {
        int i = q[h++];
        int r = rcv[i];
        if (r == i) continue;
        cnt[r] += cnt[i];
        if (--indeg[r] == 0) q[t++] = r;
    }
    int ok = (t == N) ? 0 : -1;
    free(indeg); free(q);
    return ok;
}

/* Number of cells lying on receiver cycles of length >= 2 (0 for a forest). */
int orc_count_cycle_nodes(const int32_t *rcv, int N)
{
    int32_t *indeg = (int32_t *)calloc((size_t)N, sizeof(int32_t));
    int32_t *q = (int32_t *)malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N; ++i) if (rcv[i] != i) indeg[rcv[i]]++;
    int h = 0, t = 0, selfl = 0;
    for (int i = 0; i < N; ++i) { if (rcv[i] == i) ++selfl; if (indeg[i] == 0) q[t++] = i; }
    while (h < t) {
        int i = q[h++];
        int r = rcv[i];
        if (r == i) continue;
        if (--indeg[r] == 0) q[t++] = r;
    }
    /* nodes never popped are on cycles (self-loops are roots, they pop once their donors drain) */
    int cyc = N - t;
    free(indeg); free(q);
    (void)selfl;
    return cyc;
}

/* ---- precision-generic part ---------------------------------------------- */
#define R float
#define SFX(n) n##_f32
#define KEY_T int64_t
#define KEY_LESS(a, b) ((a) < (b))
#define KEY_EQ(a, b) ((a) == (b))
#define KEY_FROM_REAL(f, i) orc_pack_float_index((f), (i))
#define REAL_FROM_KEY(k, pf, pi) key32_split((k), (pf), (pi))
#define R_MIN(a, b) fminf((a), (b))
#define R_MAX(a, b) fmaxf((a), (b))
/* h^(5/3) with the exponent rounded to f32 as Taichi folds 5./3.; evaluated in
 * double and rounded once (the correctly rounded f32 power) — the GPU kernel
 * does the same, so both sides agree bit for bit. */
#define R_POW53(h) ((float)pow((double)(h), (double)(5.0f / 3.0f)))
#define R_SQRT(x) sqrtf(x)
#include "pff_oracle_real.h"
#undef R
#undef SFX
#undef KEY_T
#undef KEY_LESS
#undef KEY_EQ
#undef KEY_FROM_REAL
#undef REAL_FROM_KEY
#undef R_MIN
#undef R_MAX
#undef R_POW53
#undef R_SQRT

#define R double
#define SFX(n) n##_f64
#define KEY_T orc_key64
#define KEY_LESS(a, b) key64_less((a), (b))
#define KEY_EQ(a, b) key64_eq((a), (b))
#define KEY_FROM_REAL(f, i) key64_make((f), (i))
#define REAL_FROM_KEY(k, pf, pi) key64_split((k), (pf), (pi))
#define R_MIN(a, b) fmin((a), (b))
#define R_MAX(a, b) fmax((a), (b))
#define R_POW53(h) pow((h), 5.0 / 3.0)
#define R_SQRT(x) sqrt(x)
#include "pff_oracle_real.h"

/* ---- whole graphflood iterations: graphflood/gf_fields.py:111-141 --------- *
 * Precision-generic driver over caller-owned state (zh, h, Q).  Parameters are
 * given in double; the f32 driver rounds each constant the way the reference's
 * Python constant folding does (e.g. PREC*DX*DX and DX**2 in double, then f32).
 * dhmax_out[n] = max |h_after - h_before| of iteration n.                      */
typedef struct {
    double dx, prec, manning, edgesw, dt, min_slope, fill_eps;
    int serial_fill;
} orc_gf_params;

#define GF_DRIVER(R, SFX, KEY_T)                                                          \
    int SFX(orc_graphflood_run)(R *zh, R *h, R *Q, const orc_grid *g, const orc_gf_params *pp, \
                                int niter, R *dhmax_out)                                  \
    {                                                                                     \
        const int N = g->nx * g->ny;                                                      \
        int32_t *rec = malloc(sizeof(int32_t) * N), *rec_ = malloc(sizeof(int32_t) * N),  \
                *rec__ = malloc(sizeof(int32_t) * N), *bid = malloc(sizeof(int32_t) * N), \
                *snode = malloc(sizeof(int32_t) * (N + 1));                               \
        R *grad = malloc(sizeof(R) * N), *zp = malloc(sizeof(R) * N),                     \
          *z_ = malloc(sizeof(R) * N), *tmp = malloc(sizeof(R) * N),                      \
          *dh = malloc(sizeof(R) * N), *h0 = malloc(sizeof(R) * N);                       \
        uint8_t *isb = calloc(N, 1), *tag = calloc(N, 1), *tag_ = calloc(N, 1);            \
        KEY_T *sad = malloc(sizeof(KEY_T) * (N + 1)), *out = malloc(sizeof(KEY_T) * (N + 1)); \
        const int nr = orc_ceil_log2(N);                                                  \
        R *inc = malloc(sizeof(R) * (nr + 1));                                            \
        for (int it = 0; it < nr; ++it) inc[it] = (R)(ldexp(1.0, it - 1) * pp->fill_eps); \
        const R dx = (R)pp->dx, dx2 = (R)(pp->dx * pp->dx),                               \
                prec_dx2 = (R)(pp->prec * pp->dx * pp->dx), man = (R)pp->manning,         \
                esw = (R)pp->edgesw, dt = (R)pp->dt, msl = (R)pp->min_slope;              \
        for (int n = 0; n < niter; ++n) {                                                 \
            memcpy(h0, h, sizeof(R) * N);                                                 \
            SFX(orc_compute_receivers)(zh, rec, grad, g, dx);                             \
            SFX(orc_reroute_flow)(bid, rec, rec_, rec__, zh, zp, isb, out, sad, snode, tag, \
                                  tag_, g, 1, NULL);                                      \
            SFX(orc_fill_z_add_delta)(zh, h, z_, rec, rec_, rec__, inc, nr, N,            \
                                      pp->serial_fill, tmp);                              \
            for (int s = 0; s < 5; ++s) SFX(orc_diffuse_q)(zh, Q, tmp, g, dx, prec_dx2);  \
            SFX(orc_graphflood_core)(h, zh, dh, rec, Q, N, dx, dx2, man, esw, dt, msl);   \
            if (dhmax_out) {                                                              \
                R m = 0;                                                                  \
                for (int i = 0; i < N; ++i) {                                             \
                    R d = h[i] - h0[i];                                                   \
                    d = d < 0 ? -d : d;                                                   \
                    if (d > m || d != d) m = d;                                           \
                }                                                                         \
                dhmax_out[n] = m;                                                         \
            }                                                                             \
        }                                                                                 \
        free(rec); free(rec_); free(rec__); free(bid); free(snode); free(grad); free(zp); \
        free(z_); free(tmp); free(dh); free(h0); free(isb); free(tag); free(tag_);        \
        free(sad); free(out); free(inc);                                                  \
        return 0;                                                                         \
    }

#define SFX32(n) n##_f32
#define SFX64(n) n##_f64
GF_DRIVER(float, SFX32, int64_t)
GF_DRIVER(double, SFX64, orc_key64)

/* ---- legacy downstream tree algorithms (archive/fastflow/kernels) ---------
 * Serial restatements; each round reads the start-of-round arrays (the
 * reference double-buffers them and copies back after every round). */

/* tree_accum_down.py:15-21, driven ceil(log2 n) times by
 * _save_fasftflow/fastflow/tree_accum_down.py:20-34: p = p + W*p[rcv],
 * W = W*W[rcv], rcv = rcv[rcv]; rcv, W and p end as the reference leaves them. */
void orc_tree_accum_down_f32(int32_t *rcv, float *W, float *p, int N, int32_t *r2, float *W2, float *p2)
{
    const int rounds = orc_ceil_log2(N);
    for (int it = 0; it < rounds; ++it) {
        for (int i = 0; i < N; ++i) {
            const int r = rcv[i];
            const float t = W[i] * p[r];
            p2[i] = p[i] + t;
            W2[i] = W[i] * W[r];
            r2[i] = rcv[r];
        }
        memcpy(rcv, r2, sizeof(int32_t) * (size_t)N);
        memcpy(W, W2, sizeof(float) * (size_t)N);
        memcpy(p, p2, sizeof(float) * (size_t)N);
    }
}

/* tree_max_down.py:7-12 driven by _save_fasftflow/fastflow/tree_max_down.py:20-31:
 * where rcv[rcv] != rcv, p = max(p[rcv], p) and rcv = rcv[rcv]; other nodes keep
 * their values.  max(a, b) is taken as a > b ? a : b. */
void orc_tree_max_down_f32(int32_t *rcv, float *p, int N, int32_t *r2, float *p2)
{
    const int rounds = orc_ceil_log2(N);
    for (int it = 0; it < rounds; ++it) {
        for (int i = 0; i < N; ++i) {
            const int r = rcv[i];
            if (rcv[r] != r) {
                const float a = p[r], b = p[i];
                p2[i] = a > b ? a : b;
                r2[i] = rcv[r];
            } else {
                p2[i] = p[i];
                r2[i] = r;
            }
        }
        memcpy(rcv, r2, sizeof(int32_t) * (size_t)N);
        memcpy(p, p2, sizeof(float) * (size_t)N);
    }
}

/* erode_deposit.py:7-24 (deposition, implicit stream-power factors), then the
 * downstream solve of _archived/erode_deposit.py:30-39: tree_accum_down on
 * (rcv, We, pe).  z is updated by the deposition in place; pe ends as the new
 * elevations (the reference's return value), We as its jumped weights; rcv is
 * jumped in place.  Powers are taken in double and rounded once to f32. */
void orc_erode_deposit_f32(float *z, const uint8_t *bound, int32_t *rcv, const float *drain, const float *Qs,
                           float dt, float dx, float k_spl, float k_t, float k_h, float k_d, float m,
                           float *pe, float *We, int N, int32_t *r2, float *W2, float *p2)
{
    for (int i = 0; i < N; ++i) {
        if (!bound[i]) {
            const float cd = fminf(k_d / drain[i], 1.0f);
            const float dz = dt * cd;
            z[i] += dz * Qs[i];
        }
        const float pm = (float)pow((double)drain[i], (double)m);
        const float pmm = (float)pow((double)drain[i], (double)(-m));
        float s = k_spl * pm;
        s = s + k_t;
        s = s + k_h * pmm;
        const float K = (dt / dx) * s;
        pe[i] = z[i] / (1.0f + K);
        We[i] = K / (1.0f + K);
        if (bound[i]) {
            pe[i] = z[i];
            We[i] = 0.0f;
        }
    }
    orc_tree_accum_down_f32(rcv, We, pe, N, r2, W2, p2);
}
