/*
 * CPU oracle — precision-generic part (included twice by pff_oracle.c, once with
 * R = float for the parity oracle and once with R = double for the FP64 run of
 * the same update).  TEST INFRASTRUCTURE ONLY: tests, the smoke check and the
 * bench's CPU-baseline leg use it as the checker; the product never calls it.
 *
 * Semantics = serial ascending-index execution of every top-level loop of the
 * reference's Taichi kernels (Taichi CPU backend with one thread): last writer
 * wins, in-place reads see earlier writes of the same loop.  Exceptions, pinned
 * because the reference is racy there on its own GPU backend:
 *   - topofill round: SNAPSHOT reads of z_ (all reads of a round before any
 *     write); the serial-ascending variant is kept as topofill_round_serial for
 *     measuring the difference (fill_topo.py:17-45).
 * Every function cites the reference file:line it restates (paths relative to
 * the pyfastflow project root).
 *
 * Expected macros: R (float|double), SFX(name), KEY_T, KEY_LESS, KEY_EQ,
 * KEY_FROM_REAL, REAL_FROM_KEY, R_MIN, R_MAX,
 * R_POW53 (h^(5/3) in R), R_SQRT.
 */

/* ---- D4 steepest-descent receivers: flow/receivers.py:31-58 ---------------- */
void SFX(orc_compute_receivers)(const R *z, int32_t *rcv, R *grad, const orc_grid *g, R dx)
{
    const int N = g->nx * g->ny;
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        int r = i;            /* receivers.py:33 */
        R sr = (R)0;          /* receivers.py:34 */
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, i, k);
            if (j == -1) continue;            /* tsr = -1 never beats sr >= 0 */
            R tsr = (z[i] - z[j]) / dx;       /* receivers.py:43, IEEE division */
            if (tsr > sr) { sr = tsr; r = j; } /* strict '>' : first k wins ties (:50-52) */
        }
        rcv[i] = r;
        grad[i] = sr;
    }
}

/* ---- saddlesort: flow/lakeflow.py:106-281 ---------------------------------- *
 * Basin arrays (basin_saddle, outlet, saddlenode) have nb = N+1 entries so that
 * basin id N (custom mode, last cell interior) is in bounds; the reference sizes
 * them N and would read out of bounds there (lakeflow.py:194,228).           */
void SFX(orc_saddlesort)(const int32_t *bid, uint8_t *is_border, R *zp,
                         KEY_T *saddle, int32_t *snode, KEY_T *outlet,
                         const R *z, const orc_grid *g)
{
    const int N = g->nx * g->ny;
    const KEY_T invalid = KEY_FROM_REAL((R)1e8f, 42);   /* lakeflow.py:127 */
    /* pass 1: borders and z' (:132-157) */
    for (int i = 0; i < N; ++i) {
        if (orc_can_leave(g, i)) { zp[i] = z[i]; continue; }
        is_border[i] = 0;
        zp[i] = (R)1e9f;
        R zn = (R)1e9f;
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, i, k);
            if (j == -1) continue;
            if (bid[j] != bid[i]) { is_border[i] = 1; zn = R_MIN(zn, z[j]); }
        }
        if (is_border[i]) zp[i] = R_MAX(z[i], zn);
    }
    /* pass 2: init (:164-167) then per-basin minimum saddle key (:170-194) */
    for (int i = 0; i < N; ++i) { saddle[i] = invalid; outlet[i] = invalid; snode[i] = -1; }
    saddle[N] = invalid; outlet[N] = invalid; snode[N] = -1;
    for (int i = 0; i < N; ++i) {
        if (!is_border[i]) continue;
        int tb = bid[i];
        KEY_T res = invalid;
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, i, k);
            if (j == -1) continue;
            if (bid[j] != tb) {
                KEY_T c = KEY_FROM_REAL(zp[i], bid[j]);
                if (KEY_LESS(c, res)) res = c;
            }
        }
        if (KEY_EQ(res, invalid)) continue;
        if (KEY_LESS(res, saddle[tb])) saddle[tb] = res;
    }
    /* pass 3: saddle node, serial last writer = largest cell index (:199-219) */
    for (int i = 0; i < N; ++i) {
        if (!is_border[i] || bid[i] == 0) continue;
        R tz; int tb;
        REAL_FROM_KEY(saddle[bid[i]], &tz, &tb);
        int ishere = 0;
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, i, k);
            if (j == -1) continue;
            if (bid[j] == tb && zp[i] == tz) ishere = 1;
        }
        if (ishere) snode[bid[i]] = i;
    }
    /* pass 4: outlet = lowest foreign neighbour of the saddle node (:226-250) */
    for (int b = 1; b < N; ++b) {
        if (KEY_EQ(saddle[b], invalid)) continue;
        int node = snode[b];
        if (node < 0) continue;  /* unreachable for finite z (a key always has its node) */
        R tz = (R)1e9f;
        int r = -1;
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, node, k);
            if (j == -1) continue;
            if (bid[j] != b && tz > z[j]) { tz = z[j]; r = j; }
        }
        if (r > -1) {
            KEY_T c = KEY_FROM_REAL(tz, r);
            if (KEY_LESS(c, outlet[b])) outlet[b] = c;
        }
    }
    /* pass 5: 2-cycle removal, serial in place (:255-281) */
    for (int b = 1; b < N; ++b) {
        if (KEY_EQ(outlet[b], invalid)) continue;
        R t; int ro, ro2;
        REAL_FROM_KEY(outlet[b], &t, &ro);
        int bd1 = bid[ro];
        if (bd1 == 0) continue;
        REAL_FROM_KEY(outlet[bd1], &t, &ro2);   /* invalid key unpacks to index 42 */
        int bd2 = (ro2 >= 0 && ro2 < N) ? bid[ro2] : -1;  /* N <= 42: no basin matches */
        if (bd2 == b && bd1 < b) {
            outlet[b] = invalid; saddle[b] = invalid; snode[b] = -1;
        }
    }
}

/* ---- reroute_flow: flow/lakeflow.py:466-538 (carve :405-438, jump :285-304) -- */
int SFX(orc_reroute_flow)(int32_t *bid, int32_t *rec, int32_t *rec_, int32_t *rec__,
                          const R *z, R *zp, uint8_t *is_border, KEY_T *outlet,
                          KEY_T *saddle, int32_t *snode, uint8_t *tag, uint8_t *tag_,
                          const orc_grid *g, int carve, int *n_outer_out)
{
    const int N = g->nx * g->ny;
    const KEY_T invalid = KEY_FROM_REAL((R)1e8f, 42);
    memcpy(rec_, rec, sizeof(int32_t) * (size_t)N);           /* :491 */
    int Ndep = orc_depression_counter(rec, g);                /* :493 */
    int n_outer = 0;
    if (Ndep == 0) { if (n_outer_out) *n_outer_out = 0; return 0; }
    const int outer = orc_ceil_log2(Ndep) + 1;                /* :500 */
    const int nprop = orc_ceil_log2(N) + 1;                   /* :510 */
    for (int it = 0; it < outer; ++it) {
        int Ndep_bis = orc_depression_counter(rec_, g);       /* :501 */
        orc_basin_id_init(bid, g);                            /* :507 */
        memcpy(rec__, rec_, sizeof(int32_t) * (size_t)N);     /* :508 */
        for (int p = 0; p < nprop; ++p) orc_propagate_basin(bid, rec__, N);
        ++n_outer;
        if (Ndep_bis == 0) break;                             /* :512 */
        SFX(orc_saddlesort)(bid, is_border, zp, saddle, snode, outlet, z, g);
        if (carve) {
            /* reroute_carve :424-438 */
            for (int i = 0; i < N; ++i) tag[i] = 0;
            for (int i = 0; i < N; ++i) if (snode[i] != -1) tag[snode[i]] = 1;
            memcpy(tag_, tag, (size_t)N);
            memcpy(rec, rec_, sizeof(int32_t) * (size_t)N);
            memcpy(rec__, rec_, sizeof(int32_t) * (size_t)N);
            int change = 1;
            while (change) {                                  /* :431-435 */
                change = 0;
                for (int i = 0; i < N; ++i) {                 /* iteration pass 1 :355-359 */
                    if (tag[i]) tag_[rec[i]] = 1;
                    rec_[i] = rec[i];
                }
                for (int i = 0; i < N; ++i) {                 /* pass 2 :362-368 */
                    rec[i] = rec_[rec_[i]];
                    if (tag[i] != tag_[i]) change = 1;
                    tag[i] = tag_[i];
                }
            }
            /* finalise_reroute_carve(rec, rec__, ...) :390-403 */
            for (int i = 0; i < N; ++i) rec[i] = rec__[i];
            for (int i = 0; i < N; ++i)
                if (tag[rec__[i]] && tag[i] && i != rec__[i]) rec[rec__[i]] = i;
            for (int i = 0; i < N; ++i) {
                if (KEY_EQ(outlet[i], invalid)) continue;
                R t; int node;
                REAL_FROM_KEY(outlet[i], &t, &node);
                rec[snode[i]] = node;
            }
            memcpy(rec_, rec, sizeof(int32_t) * (size_t)N);   /* :526 */
        } else {
            for (int i = 0; i < N; ++i) {                     /* reroute_jump :299-304 */
                if (KEY_EQ(outlet[i], invalid)) continue;
                R t; int node;
                REAL_FROM_KEY(outlet[i], &t, &node);
                rec_[i - 1] = node;
            }
        }
    }
    orc_basin_id_init(bid, g);                                /* :537 */
    if (n_outer_out) *n_outer_out = n_outer;
    return Ndep;
}

/* ---- one fill round: flow/fill_topo.py:17-45 ------------------------------- *
 * Snapshot semantics: every read of z_ sees the value at the start of the round
 * (zs = copy of z_ taken by the caller).                                      */
static void SFX(topofill_round_snapshot)(const R *zh, R *z_, const R *zs, int32_t *rec_,
                                         int32_t *rec__, R inc, int N)
{
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        int r = rec_[i];
        rec__[i] = rec_[r];                                           /* :29 */
        if (i == r || (zs[i] > zh[r] && rec_[r] == r)) continue;      /* :32 */
        z_[i] = R_MAX(zs[i], zs[r] + inc);                            /* :36 */
    }
    OMP_FOR
    for (int i = 0; i < N; ++i) rec_[i] = rec__[i];                   /* :39-40 */
}

/* Serial ascending-index variant of the same round (Taichi CPU, one thread). */
static void SFX(topofill_round_serial)(const R *zh, R *z_, int32_t *rec_, int32_t *rec__,
                                       R inc, int N)
{
    for (int i = 0; i < N; ++i) {
        int r = rec_[i];
        rec__[i] = rec_[r];
        if (i == r || (z_[i] > zh[r] && rec_[r] == r)) continue;
        z_[i] = R_MAX(z_[i], z_[r] + inc);
    }
    for (int i = 0; i < N; ++i) rec_[i] = rec__[i];
}

/* fill_z_add_delta: flow/fill_topo.py:99-125 (with _apply_fill_z_add_delta :82-97).
 * inc[it] = float(2^(it-1) * epsilon) per round, it = 0..ceil(log2 N)-1,
 * computed by the caller exactly as the reference's Python constant folding. */
void SFX(orc_fill_z_add_delta)(R *zh, R *h, R *z_, const int32_t *rec, int32_t *rec_,
                               int32_t *rec__, const R *inc, int nrounds, int N,
                               int serial, R *scratch)
{
    memcpy(z_, zh, sizeof(R) * (size_t)N);
    memcpy(rec_, rec, sizeof(int32_t) * (size_t)N);
    memcpy(rec__, rec, sizeof(int32_t) * (size_t)N);
    for (int it = 0; it < nrounds; ++it) {
        if (serial) {
            SFX(topofill_round_serial)(zh, z_, rec_, rec__, inc[it], N);
        } else {
            memcpy(scratch, z_, sizeof(R) * (size_t)N);
            SFX(topofill_round_snapshot)(zh, z_, scratch, rec_, rec__, inc[it], N);
        }
    }
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        R d = z_[i] - zh[i];
        h[i] += d;
        zh[i] = z_[i];
    }
}

/* ---- MFD discharge diffusion: graphflood/gf_hydrodynamics.py:24-75 --------- *
 * temp[j] accumulates in ascending source index, then k order (serial atomics);
 * the j == -1 target of the reference (an out-of-bounds add of 0) is skipped. */
void SFX(orc_diffuse_q)(const R *zh, R *Q, R *temp, const orc_grid *g, R dx, R prec_dx2)
{
    const int N = g->nx * g->ny;
    for (int i = 0; i < N; ++i) {
        temp[i] = prec_dx2;
        if (orc_can_leave(g, i)) Q[i] = (R)0;
    }
    for (int i = 0; i < N; ++i) {
        if (orc_can_leave(g, i)) continue;
        R sums = (R)0;
        int js[4];
        for (int k = 0; k < 4; ++k) {
            int j = orc_neighbour(g, i, k);
            js[k] = j;
            sums += R_MAX((R)0, (j != -1) ? (zh[i] - zh[j]) / dx : (R)0);
        }
        if (sums == (R)0) continue;
        for (int k = 0; k < 4; ++k) {
            int j = js[k];
            if (j == -1) continue;
            R tS = R_MAX((R)0, (zh[i] - zh[j]) / dx);
            R w = tS / sums;
            temp[j] += w * Q[i];
        }
    }
    for (int i = 0; i < N; ++i) Q[i] = temp[i];
}

/* ---- Manning depth update: graphflood/gf_hydrodynamics.py:79-129 ----------- */
void SFX(orc_graphflood_core)(R *h, R *zh, R *dh, const int32_t *rec, const R *Q, int N,
                              R dx, R dx2, R manning, R edgesw, R dt, R min_slope)
{
    OMP_FOR
    for (int i = 0; i < N; ++i) {
        R tS = edgesw;
        if (rec[i] != i) tS = R_MAX((zh[i] - zh[rec[i]]) / dx, min_slope);
        R Qo = dx * R_POW53(h[i]);
        Qo = Qo / manning;
        Qo = Qo * R_SQRT(tS);
        R tdh = (Q[i] - Qo) / dx2;
        tdh = tdh * dt;
        h[i] += tdh;
        if (h[i] < (R)0) tdh += h[i];
        dh[i] = tdh;
    }
    OMP_FOR
    for (int i = 0; i < N; ++i) { h[i] += dh[i]; zh[i] += dh[i]; }
}
