/*
 * libpff — B200 (sm_100a) flow routing and GraphFlood hot path, C ABI.
 *
 * Every entry point takes plain device pointers (CUDA global memory), sizes, and
 * a CUDA stream (cudaStream_t passed as void*; NULL = legacy default stream).
 * Nothing here allocates device memory except where a call says so: scratch is a
 * caller-provided device buffer whose size the matching *_workspace_bytes()
 * query returns.  Calls are asynchronous on `stream` unless documented as
 * returning a host-visible count (those synchronize the stream).
 *
 * Status: 0 = PFF_OK; on error the call returns a nonzero PFF_ERR_* code and
 * pff_last_error_string() describes it (per host thread).  No call aborts,
 * prints or traps.
 *
 * Grid arguments restate pyfastflow's compile-time globals (pyfastflow/constants.py:
 * NX :31, NY :34, DX :28, BOUND_MODE :50, boundaries :53) as runtime values:
 *   nx, ny      grid columns / rows (nx, ny >= 2), cells are row-major i = row*nx + col
 *   dx          cell size
 *   bound_mode  0 normal, 1 periodic east-west, 2 periodic north-south, 3 custom
 *   codes       N uint8 boundary codes (device), custom mode only, else NULL
 *               (0 nodata, 1 normal, 3 outlet, 7 inlet, 9 periodic)
 * Receivers are int32 cell indices; basin arrays (basin_saddle, outlet,
 * basin_saddlenode) have N+1 entries.
 */
#ifndef PFF_H
#define PFF_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFF_OK 0
#define PFF_ERR_ARG 1        /* invalid argument (size, pointer, mode) */
#define PFF_ERR_CUDA 2       /* CUDA runtime error (launch or copy) */
#define PFF_ERR_NOCONV 3     /* iteration cap reached before convergence */
#define PFF_ERR_WORKSPACE 4  /* workspace too small */
#define PFF_ERR_UNAVAILABLE 5 /* this path is not available here (e.g. CUDA graphs switched off) */

/* Library version (major*10000 + minor*100 + patch). */
int pff_version(void);
/* Description of the last error on the calling host thread ("" if none). */
const char *pff_last_error_string(void);
/* Total number of CUDA kernels this library has launched in this process (no
 * counterpart in the reference: used to report GPU launches per step). */
long long pff_launch_count(void);
/* Kernel timing probes (no reference counterpart; used by benchmarks to time the
 * dominant kernels inside a call).  pff_probe_enable(1) clears and arms them: each
 * probed launch made outside stream capture is then bracketed by two CUDA events on
 * its own stream (at most 512 launches per kernel name).  pff_probe_enable(0)
 * disarms and clears.  pff_probe_read waits for the recorded events of the kernel
 * named `name` (for example "k_tree_tile<up>") and returns their summed event time
 * in milliseconds and the number of probed launches (0 if it never ran). */
int pff_probe_enable(int on);
int pff_probe_read(const char *name, double *total_ms, int *launches);
/* Whether pff_reroute_flow drives its outer loop from a device-side CUDA graph
 * (1, the default) or from the host (0: one synchronisation per outer iteration;
 * its kernels can then be profiled and probed one by one).  The environment
 * variable PFF_REROUTE_NO_GRAPH makes 0 the default.  Returns the previous
 * setting.  No reference counterpart. */
int pff_reroute_use_graphs(int on);
/* Make `device` current for this library's calls on the calling host thread
 * (the library links its own CUDA runtime; callers that use several GPUs set
 * the device that owns the buffers before calling).  No reference counterpart. */
int pff_set_device(int device);

/* ---- receivers --------------------------------------------------------------
 * Replaces pyfastflow/flow/receivers.py:15-58 compute_receivers(z, receivers,
 * gradient): D4 steepest descent, strict '>' (first direction k wins ties),
 * IEEE f32 (z[i]-z[j])/dx; self-receiver for pits and flats. */
int pff_compute_receivers(const float *z, int32_t *receivers, float *gradient, int nx, int ny,
                          float dx, int bound_mode, const uint8_t *codes, void *stream);

/* receivers.py:46-47 with RAND_RCV: every direction's slope (or -1 if the neighbour
 * is invalid) is multiplied by u in [0, 1) before the same strict '>' selection; the
 * gradient is the chosen scaled slope.  u = (SplitMix64(seed ^ SplitMix64(4*i + k))
 * >> 40) / 2^24: reproducible for a seed; the reference's draws (Taichi's generator)
 * are not, so parity is statistical. */
int pff_compute_receivers_stochastic(const float *z, int32_t *receivers, float *gradient, int nx, int ny,
                                     float dx, int bound_mode, const uint8_t *codes,
                                     unsigned long long seed, void *stream);

/* Which kernel pff_compute_receivers uses in modes 0-2 when nx % 4 == 0 and the
 * arrays are 16-byte aligned: 1 (default) the lean kernel (one Markstein-corrected
 * quotient per cell, drops shared between neighbours, edges on the same path) at
 * 7 CTAs per SM, 2 the same at 8 CTAs per SM, 0 the earlier 4-column row walk.
 * Results are identical.  Returns the previous setting.  No reference counterpart.
 * pff_receivers_div_selfcheck: runs the lean kernel's quotient for cell size dx on
 * every float in its exact range and counts the results that differ from the IEEE
 * division (must be 0); *checked = how many floats were run.  Synchronous; a
 * self-test, no reference counterpart. */
int pff_receivers_set_path(int lean);
int pff_receivers_div_selfcheck(float dx, long long *mismatches, long long *checked);

/* ---- accumulation (rake and compress) ----------------------------------------
 * Kernel-level mirrors of pyfastflow/flow/downstream_propag.py with identical
 * semantics (donor slots in ascending donor index, as the reference's serial
 * order gives):
 *   rcv2donor            downstream_propag.py:77-96   (ndnr must be zero on entry)
 *   rake_compress_accum  downstream_propag.py:99-179  (one round)
 *   fuse                 downstream_propag.py:59-74 */
int pff_rcv2donor(const int32_t *rcv, int32_t *dnr, int32_t *ndnr, int N, void *stream);
int pff_rake_compress_accum(int32_t *dnr, int32_t *ndnr, float *p, int32_t *src, int32_t *dnr_,
                            int32_t *ndnr_, float *p_, int iteration, int N, void *stream);
int pff_fuse(float *A, const int32_t *src, const float *B, int iteration, int N, void *stream);

/* Whole accumulation as FlowRouter.accumulate_constant_Q drives it
 * (pyfastflow/flow/flowfields.py:254-292), for any receiver forest:
 *   Q      in: per-cell seed (value*dx^2, 1, or per-cell weights); out: upstream sum,
 *          bit-identical to the reference's f32 rake-and-compress result
 *   counts out (optional, may be NULL): exact uint32 upstream cell counts
 * workspace: pff_accumulate_workspace_bytes(N) bytes of device scratch.
 * A node with more than 4 donors (only jump rerouting can produce one; the
 * reference's slots overflow there, downstream_propag.py:94-96) is reported as
 * PFF_ERR_ARG.  Synchronizes `stream` once at the end to read that check. */
size_t pff_accumulate_workspace_bytes(int N);
int pff_accumulate(const int32_t *receivers, float *Q, uint32_t *counts, int N, void *workspace,
                   size_t workspace_bytes, void *stream);
/* Same, with the grid given: donor lists are then built by a gather over each
 * cell's D4 neighbours (no atomics); receivers that are not D4 neighbours are
 * detected on the device and handled by the general path.  Same results. */
int pff_accumulate_grid(const int32_t *receivers, float *Q, uint32_t *counts, int nx, int ny,
                        int bound_mode, const uint8_t *codes, int N, void *workspace,
                        size_t workspace_bytes, void *stream);
/* Tuning switch of pff_accumulate_grid (no reference counterpart): the number of
 * leading rounds (3 default, 4, or 0 = off) run per spatial tile in shared memory
 * for boundary modes 0-2 on grids of at least 3 x 3.  Every setting gives the same
 * results.  Process-wide; returns PFF_ERR_ARG for other values. */
int pff_accumulate_set_front(int rounds);

/* Drainage accumulation by hierarchical tile contraction, for any receiver forest
 * (any in-degree: the jump rerouting of lakeflow.py:285-304, whose pits can gain
 * more than 4 donors, is handled).  Replaces the whole accumulate_constant_Q chain
 * of pyfastflow/flow/flowfields.py:254-292 (rcv2donor + rake_compress_accum + fuse,
 * downstream_propag.py:21-179) with exact sums:
 *   counts  out (optional): uint32 number of cells upstream of each cell, itself
 *           included -- identical to the reference's counts;
 *   Q       out (optional): the upstream sum of the seeds (weights[i], or `value`
 *           for every cell if weights is NULL) formed exactly in 64-bit fixed point
 *           (seed * 2^s, s chosen from max|seed| * N) and rounded once to f32.  The
 *           reference's f32 sums carry their own rounding; Q differs from them by
 *           that rounding only.  Seeds smaller than max|seed| * N * 2^-62 lose
 *           their low bits.  Q may alias weights.  Deterministic.
 *   local   1 if every receiver is the cell itself or a D4 neighbour (periodic
 *           wrap included) -- the output of compute_receivers and of carve
 *           rerouting; 0 for any receivers (each 32 x 32 tile may then have at most
 *           256 cells whose receiver is outside it).
 * Asynchronous (no host synchronisation).  Problems are recorded in a status word
 * read by pff_accumulate_tree_status (synchronizes `stream`): 1 receiver out of
 * range, 2 receiver cycle, 4 a tile with too many exits, 8 local = 1 violated,
 * 16 non-finite seed; Q and counts are unspecified when it is nonzero.
 * workspace: pff_accumulate_tree_workspace_bytes(nx, ny, local) bytes. */
size_t pff_accumulate_tree_workspace_bytes(int nx, int ny, int local);
int pff_accumulate_tree(const int32_t *receivers, const float *weights, float value, float *Q,
                        uint32_t *counts, int nx, int ny, int local, void *workspace,
                        size_t workspace_bytes, void *stream);
int pff_accumulate_tree_status(int nx, int ny, int local, void *workspace, size_t workspace_bytes,
                               int *status, void *stream);

/* ---- lake / depression rerouting -----------------------------------------------
 * Replaces pyfastflow/flow/lakeflow.py:466-538 reroute_flow(bid, rec, rec_, rec__,
 * z, z_prime, is_border, outlet, basin_saddle, basin_saddlenode, tag, tag_,
 * change, carve).  Same buffers and meaning; rec is rerouted in place (carve) or
 * the result is left in rec_ (carve = 0, as the reference leaves it).  is_border,
 * tag, tag_ are uint8 (0/1).  bid ends in the basin_id_init state, as in the
 * reference.  Synchronizes `stream` (reads pit counts on the host, like the
 * reference's depression_counter).  n_outer_out (host, optional) receives the
 * number of outer iterations run.  workspace: pff_reroute_workspace_bytes(N). */
size_t pff_reroute_workspace_bytes(int N);
int pff_reroute_flow(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                     float *z_prime, uint8_t *is_border, int64_t *outlet, int64_t *basin_saddle,
                     int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int carve, int nx,
                     int ny, int bound_mode, const uint8_t *codes, void *workspace,
                     size_t workspace_bytes, int *n_outer_out, void *stream);
/* pff_reroute_flow (carve) split at its one host synchronisation, so that a caller can
 * queue more work behind the reroute before it looks at the result (no reference
 * counterpart; the Flooder's pipelined loop uses it).
 *   - pff_reroute_flow_async launches the device-driven outer loop and returns; the
 *     graph's last node copies its final state (9 ints) into ctl_out (device memory, or
 *     pinned host memory, which it writes through its unified address).
 *     Returns PFF_ERR_UNAVAILABLE where that loop cannot run (graphs switched off by
 *     pff_reroute_use_graphs / PFF_REROUTE_NO_GRAPH, or not supported).
 *   - pff_reroute_flow_finish takes a host copy of those 9 ints, once the launch has
 *     completed, and does what pff_reroute_flow does after its graph: nothing if the
 *     loop finished on the device (ctl[3] = 1 no pits, or 2 done), the reference's
 *     steps on the host if it stopped for them (3, 4; synchronises), an error
 *     otherwise.  Same buffers and workspace as the async call; *n_outer_out as in
 *     pff_reroute_flow.
 * Together they leave every buffer as one pff_reroute_flow(carve = 1) call does. */
int pff_reroute_flow_async(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                           float *z_prime, uint8_t *is_border, int64_t *outlet, int64_t *basin_saddle,
                           int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int nx, int ny,
                           int bound_mode, const uint8_t *codes, void *workspace, size_t workspace_bytes,
                           int *ctl_out, void *stream);
int pff_reroute_flow_finish(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__, const float *z,
                            float *z_prime, uint8_t *is_border, int64_t *outlet, int64_t *basin_saddle,
                            int32_t *basin_saddlenode, uint8_t *tag, uint8_t *tag_, int nx, int ny,
                            int bound_mode, const uint8_t *codes, void *workspace, size_t workspace_bytes,
                            const int *ctl_host, int *n_outer_out, void *stream);
/* A region of work that runs only after a finished asynchronous reroute (no reference
 * counterpart).  pff_guard_begin starts capturing `stream` (not the legacy default
 * stream) into the body of a conditional graph; everything the caller issues on it
 * until pff_guard_end is recorded, not run.  pff_guard_launch runs the graph: its
 * first node reads ctl[3] (the state words of pff_reroute_flow_async) and the
 * optional flag, and the body runs when the state is 1 or 2 and *flag is 0.
 * pff_guard_destroy frees it.  At most 1024 regions at a time. */
int pff_guard_begin(const int *ctl, const int *flag, void *stream, int *id);
int pff_guard_end(int id, void *stream);
int pff_guard_launch(int id, void *stream);
int pff_guard_destroy(int id);
/* out_dev[0] and out_host[0] = val[0], each if non-NULL: one small kernel; out_host may be
 * pinned host memory (written through its unified address, no copy engine). */
int pff_value_store(const float *val, float *out_dev, float *out_host, void *stream);
/* flag[0] = 1 if (double)val[0] / div < thr, else 0 (device values; the host's
 * residual test float(value) / dt < threshold made on the device, in double). */
int pff_residual_flag(const float *val, double div, double thr, int *flag, void *stream);

/* Basin labels of a receiver forest: lakeflow.py:82-101 basin_identification
 * (bid = root+1, or 0 when the root can leave the domain).  rec_ is scratch (N). */
int pff_basin_identification(int32_t *bid, const int32_t *rec, int32_t *rec_, int nx, int ny,
                             int bound_mode, const uint8_t *codes, void *stream);

/* lakeflow.py:25-44 depression_counter; writes the count to *count_out (host).
 * Synchronizes `stream`. */
int pff_depression_counter(const int32_t *rec, int nx, int ny, int bound_mode,
                           const uint8_t *codes, int *count_out, void *stream);

/* lakeflow.py:106-281 saddlesort (passes 1-5). */
int pff_saddlesort(const int32_t *bid, uint8_t *is_border, float *z_prime, int64_t *basin_saddle,
                   int32_t *basin_saddlenode, int64_t *outlet, const float *z, int nx, int ny,
                   int bound_mode, const uint8_t *codes, void *stream);

/* ---- GraphFlood ----------------------------------------------------------------
 * pyfastflow/flow/fill_topo.py:99-125 fill_z_add_delta(zh, h, z_, receivers,
 * receivers_, receivers__, epsilon): ceil(log2 N) pointer-jumping fill rounds
 * with increment float(2^(it-1)*epsilon), then h += z_-zh, zh = z_.  The round's
 * in-place read of z_ (a race in the reference) is pinned to snapshot semantics:
 * every read of a round sees the start-of-round value.  workspace:
 * pff_fill_workspace_bytes(N) bytes. */
size_t pff_fill_workspace_bytes(int N);
int pff_fill_z_add_delta(float *zh, float *h, float *z_, const int32_t *receivers,
                         int32_t *receivers_, int32_t *receivers__, double epsilon, int N,
                         void *workspace, size_t workspace_bytes, void *stream);

/* pyfastflow/flow/fill_topo.py:48-78 topofill(flow_field, epsilon, custom_z): the
 * same rounds on z with increments float(2^it * epsilon), it = 0..ceil(log2 N)-1,
 * into z_ (snapshot semantics as above); write_back = 1 then copies z_ into z (the
 * reference's default), 0 leaves z untouched (its custom_z form, z_ = custom_z).
 * No depth update.  workspace: pff_fill_workspace_bytes(N) bytes. */
int pff_topofill(float *z, float *z_, const int32_t *receivers, int32_t *receivers_, int32_t *receivers__,
                 double epsilon, int N, int write_back, void *workspace, size_t workspace_bytes, void *stream);

/* The same fill for callers that cannot allocate device memory (no workspace
 * argument): its scratch is a 16 MiB device array built into the library,
 * held on every GPU that loads the library until exit.  No counterpart in the
 * reference.  Limits and rules:
 *   - N <= PFF_NOALLOC_MAX_CELLS, else PFF_ERR_ARG;
 *   - the first call on a device looks up that array's device address, so make
 *     the first call on each device before any stream capture;
 *   - calls share the one array: calls that overlap on the GPU (other streams,
 *     other host threads) race and must be serialised by the caller.
 * Never calls cudaMalloc/cudaFree.  Same results as pff_fill_z_add_delta. */
#define PFF_NOALLOC_MAX_CELLS (1 << 22)
int pff_fill_z_add_delta_noalloc(float *zh, float *h, float *z_, const int32_t *receivers,
                                 int32_t *receivers_, int32_t *receivers__, double epsilon, int N,
                                 void *stream);

/* graphflood/gf_hydrodynamics.py:24-75 diffuse_Q_constant_prec(zh, Q, temp), run
 * `nsweeps` times (the Flooder runs 5).  prec_dx2 = float(PREC*DX*DX).  Sums are
 * formed in the reference's serial order (ascending source cell, then k), so the
 * result is deterministic.  temp: N floats (ends equal to Q, as in the reference);
 * workspace: pff_diffuse_workspace_bytes(N). */
size_t pff_diffuse_workspace_bytes(int N);
int pff_diffuse_q(const float *zh, float *Q, float *temp, int nsweeps, int nx, int ny, float dx,
                  float prec_dx2, int bound_mode, const uint8_t *codes, void *workspace,
                  size_t workspace_bytes, void *stream);

/* graphflood/gf_hydrodynamics.py:79-129 graphflood_core_cte_mannings(h, zh, dh,
 * rec, Q) with constants dx, dx2 = float(DX**2), manning, edgesw, dt (DT_HYDRO).
 * If dhmax (device float) and h_ref (device, N) are both non-NULL, dhmax receives
 * max |h_after - h_ref| (atomically maxed into its current value; zero it first). */
int pff_graphflood_core(float *h, float *zh, float *dh, const int32_t *rec, const float *Q, int N,
                        float dx, float dx2, float manning, float edgesw, float dt,
                        const float *h_ref, float *dhmax, void *stream);
/* pff_graphflood_core in one pass, for a caller that holds a copy of zh in zf (the
 * Flooder: the fill leaves the filled surface in both z_ and zh, and nothing changes
 * either before the Manning update).  The slope reads zf, so zh is updated in the
 * same pass; results are pff_graphflood_core's, bit for bit, when zf equals zh.
 * zf must not alias zh.  Replaces the two loops of gf_hydrodynamics.py:79-129 inside
 * Flooder.run_graphflood (gf_fields.py:141). */
int pff_graphflood_core_filled(float *h, float *zh, const float *zf, float *dh, const int32_t *rec,
                               const float *Q, int N, float dx, float dx2, float manning, float edgesw,
                               float dt, const float *h_ref, float *dhmax, void *stream);

/* out[0] = max |a - b| (maxed into its current value as unsigned bits, so a NaN
 * difference wins), out[1] += sum |a - b| (f32, unspecified order).  Zero out first.
 * Used for GraphFlood's residuals (the change of h over an iteration).  No
 * reference counterpart. */
int pff_abs_diff_stats(const float *a, const float *b, int N, float *out, void *stream);

/* ---- legacy downstream tree algorithms (pyfastflow's archive) ----------------------
 * The kernels of archive/fastflow/kernels with the drivers of
 * archive/_save_fasftflow/fastflow: ceil(log2 N) pointer-jumping rounds, each
 * reading the start-of-round arrays.  rcv, W and p are updated in place as those
 * drivers leave them (rcv jumped).  Synchronize `stream` (a receiver range check).
 *   pff_tree_accum_down  tree_accum_down.py:15-21: p = p + W*p[rcv], W = W*W[rcv],
 *                        rcv = rcv[rcv] -- solves x = p + W*x[rcv] downstream;
 *   pff_tree_max_down    tree_max_down.py:7-12: where rcv[rcv] != rcv,
 *                        p = max(p[rcv], p), rcv = rcv[rcv] -- the largest value on
 *                        the downstream path, the final root's value excluded;
 *                        max(a, b) = a > b ? a : b;
 *   pff_erode_deposit    erode_deposit.py:7-24 then _archived/erode_deposit.py:30-39:
 *                        z += dt*min(k_d/drain, 1)*Qs off the boundary (bound != 0),
 *                        K = dt/dx*(k_spl*drain^m + k_t + k_h*drain^-m),
 *                        pe = z/(1+K), We = K/(1+K) (pe = z, We = 0 on the boundary),
 *                        then tree_accum_down(rcv, We, pe): pe ends as the new
 *                        elevations.  Powers are evaluated in double and rounded
 *                        once to f32.
 * workspace: pff_archive_workspace_bytes(N). */
size_t pff_archive_workspace_bytes(int N);
int pff_tree_accum_down(int32_t *rcv, float *W, float *p, int N, void *workspace, size_t workspace_bytes,
                        void *stream);
int pff_tree_max_down(int32_t *rcv, float *p, int N, void *workspace, size_t workspace_bytes, void *stream);
int pff_erode_deposit(float *z, const uint8_t *bound, int32_t *rcv, const float *drain, const float *Qs,
                      float dt, float dx, float k_spl, float k_t, float k_h, float k_d, float m, float *pe,
                      float *We, int N, void *workspace, size_t workspace_bytes, void *stream);

/* ---- Ragged batch ----------------------------------------------------------------
 * Many independent tiles (own nx, ny, dx, boundary mode 0-3) packed back to back,
 * tile t's cells at [tile_offset[t], tile_offset[t] + nx*ny) in row-major order.
 * One persistent launch runs, per tile, the chain a FlowRouter user runs tile by
 * tile: compute_receivers (receivers.py:16-58), reroute_flow(carve=True)
 * (lakeflow.py:466-538) and accumulate (flowfields.py:254-292, with a per-cell
 * seed and exact uint32 counts).  No single reference counterpart: the reference
 * routes one grid per process.  Results are bit-identical to those per-tile calls.
 *
 * pff_batch_plan: validates the tiles, fills tile_offset[ntiles] and (optional)
 * order[ntiles] (the largest-first processing order) and returns the total cell
 * count; with workspace == NULL it only does that (size query), otherwise it also
 * uploads the tile table into the workspace (synchronizes `stream`).  Errors are
 * returned negated (-PFF_ERR_*).
 * pff_batch_route: asynchronous launch on `stream`, no host synchronisation, so it
 * can be captured in a CUDA graph.  Q: per-cell seed in, upstream sum out.  codes:
 * packed uint8 boundary codes (N per tile, read for custom-mode tiles only; NULL if
 * the batch has none).
 * threads: 256, 512 or 1024 per CTA; ctas_per_sm is clamped to the occupancy.
 * pff_batch_status: error bits of the last launch (synchronizes `stream`):
 * 1 = a bad tile mode (or a custom-mode tile without codes), 8 = cells of one receiver cycle ended with
 * different serial labels, 16 = a carve did not converge. */
size_t pff_batch_workspace_bytes(long long total_cells, int ntiles);
long long pff_batch_plan(const int32_t *tile_nx, const int32_t *tile_ny, const int32_t *tile_mode,
                         const float *tile_dx, int ntiles, long long *tile_offset, int32_t *order,
                         void *workspace, size_t workspace_bytes, void *stream);
int pff_batch_route(const float *z, const uint8_t *codes, int32_t *receivers, float *gradient, float *Q,
                    uint32_t *counts, long long total_cells, int ntiles, int threads, int ctas_per_sm,
                    void *workspace, size_t workspace_bytes, void *stream);
int pff_batch_status(long long total_cells, int ntiles, void *workspace, size_t workspace_bytes,
                     int *status, void *stream);

/* GraphFlood on every tile of a planned batch, one persistent launch: each tile runs
 * Flooder iterations (gf_fields.py:126-141: receivers, carve reroute, fill with
 * delta 1e-3, 5 diffusion sweeps, Manning update) until its stop or `niter`.
 * zh (the packed DEMs), h and Q are updated in place, bit-identical to a Flooder
 * per tile.  tile_consts: 4 floats per tile in caller order -- float(dx^2),
 * float(prec*dx^2), float(manning), and the stop threshold on the iteration's
 * change of h; crit 0 stops a tile when max|dh| < threshold (the reference's
 * max|dh|/dt < tol*prec with threshold = tol*prec*dt), 1 when mean|dh| < threshold,
 * -1 never.  Per tile (caller order): iters = iterations run, residuals = the last
 * (max|dh|, mean|dh|); trace (optional): niter x (max, mean) per tile.  The mean is
 * summed in an unspecified order.  Asynchronous; status bits as pff_batch_status. */
int pff_batch_graphflood(float *zh, const uint8_t *codes, float *h, float *Q, const float *tile_consts,
                         float edgesw, float dt,
                         int niter, int crit, int32_t *iters, float *residuals, float *trace,
                         long long total_cells, int ntiles, int threads, int ctas_per_sm, void *workspace,
                         size_t workspace_bytes, void *stream);

/* ---- Warm-start network (BF16 tensor-core convolutions) ---------------------------
 * No reference counterpart: the reference has no learned component.  These serve
 * a U-Net that predicts an initial GraphFlood water depth.  Activations are NHWC
 * bf16 (uint16_t bits) rows of `cs` channels; an operand is the channel slice
 * [off, off + C) of its rows.  Weights are [Cout][9][Cin] bf16 (tap = kh*3 + kw).
 * 3x3 convolutions have stride 1 and zero padding 1; products accumulate in f32.
 *
 * pff_conv3x3_fwd: y = conv(x, w) + bias (bias f32, may be NULL), ReLU if relu,
 *   y stored as bf16 (out_f32 = 0) or f32.  Cin, csx, offx multiples of 8.
 * pff_conv3x3_wflip: wt[ci][tap][co] = w[co][8 - tap][ci]; the data gradient of a
 *   convolution is pff_conv3x3_fwd of dy with wt (Cin and Cout exchanged).
 * pff_conv3x3_wgrad: dw[co][tap*Cin + ci] += sum over pixels of dy * shifted x
 *   (f32, accumulated atomically: zero dw first).  Channels multiples of 8.
 * pff_bias_grad: db[c] += sum over pixels of dy[p][c] (C <= 256).
 * pff_relu_bwd: g = 0 where y <= 0 (y the ReLU output).
 * pff_avgpool2 / _bwd: 2x2 mean pooling (H, W of the fine grid, both even); the
 *   backward spreads dy / 4, adding to dx if accumulate.
 * pff_upsample2 / _bwd: nearest 2x upsampling (H, W of the coarse grid); the
 *   backward sums each 2x2 block.
 * pff_mse_loss: loss += scale * sum w (pred - t)^2 over pred channel 0 (rows of csp
 *   floats; weight may be NULL), dpred rows (csd bf16) = (2 w (pred - t) scale, 0...).
 * pff_adam: Adam with decoupled weight decay, step >= 1; writes the bf16 copy if
 *   p_bf16 is not NULL.
 * pff_unet_features: 8-channel bf16 input rows for B tiles of N cells from the
 *   elevation, steepest slope, drainage counts, per-tile rainfall and Manning n;
 *   stats receives each tile's elevation mean and 1/std (2 floats per tile).
 * pff_unet_h0: h0 = max(exp(min(pred, 5)) - eps, 0), and the water surface zh = z + h0 if zh is
 *   not NULL; pff_unet_target: log(max(h,0) + eps). */
int pff_conv3x3_fwd(const uint16_t *x, int csx, int offx, const uint16_t *w, const float *bias, void *y,
                    int csy, int offy, int B, int H, int W, int Cin, int Cout, int relu, int out_f32,
                    void *stream);
/* Which kernel pff_conv3x3_fwd uses: 0 automatic (tcgen05 when Cin, Cout, the input
 * offset are multiples of 64 and a 128-pixel block tiles the image, else mma.sync),
 * 1 mma.sync only, 2 tcgen05 only (PFF_ERR_ARG if unsupported).  Default 0.
 * pff_conv_tc_status: 1 if a tcgen05 launch since the last call gave up waiting on
 * its pipeline (results then unspecified), else 0; synchronizes the device. */
int pff_conv_set_path(int path);
int pff_conv_tc_status(int *flag);
int pff_conv3x3_wflip(const uint16_t *w, uint16_t *wt, int Cin, int Cout, void *stream);
int pff_conv3x3_wgrad(const uint16_t *x, int csx, int offx, const uint16_t *dy, int csd, int offd, float *dw,
                      int B, int H, int W, int Cin, int Cout, void *stream);
int pff_bias_grad(const uint16_t *dy, int cs, int off, float *db, long long P, int C, void *stream);
int pff_relu_bwd(uint16_t *g, int csg, int offg, const uint16_t *y, int csy, int offy, long long P, int C,
                 void *stream);
int pff_avgpool2(const uint16_t *x, int csx, int offx, uint16_t *y, int csy, int offy, int B, int H, int W,
                 int C, void *stream);
int pff_avgpool2_bwd(const uint16_t *dy, int csd, int offd, uint16_t *dx, int csx, int offx, int B, int H,
                     int W, int C, int accumulate, void *stream);
int pff_upsample2(const uint16_t *x, int csx, int offx, uint16_t *y, int csy, int offy, int B, int H, int W,
                  int C, void *stream);
int pff_upsample2_bwd(const uint16_t *dy, int csd, int offd, uint16_t *dx, int csx, int offx, int B, int H,
                      int W, int C, void *stream);
int pff_mse_loss(const float *pred, int csp, const float *target, const float *weight, long long P,
                 uint16_t *dpred, int csd, float scale, float *loss, void *stream);
int pff_adam(float *p, const float *g, float *m, float *v, uint16_t *p_bf16, long long n, float lr, float b1,
             float b2, float eps, int step, float weight_decay, void *stream);
int pff_f32_to_bf16(const float *src, uint16_t *dst, long long n, void *stream);
int pff_unet_features(const float *z, const float *slope, const uint32_t *counts, const float *prec,
                      const float *manning, float dx, int B, long long N, float *stats, uint16_t *out,
                      void *stream);
int pff_unet_h0(const float *pred, int cs, float *h0, long long P, float eps, const float *z, float *zh,
                void *stream);
int pff_unet_target(const float *h, float *target, long long P, float eps, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PFF_H */
