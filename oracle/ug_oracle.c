/* ug_oracle.c -- TEST INFRASTRUCTURE ONLY (see ug_oracle.h).
 *
 * Plain-C restatement of the reference packing path:
 *   RNG          xoshiro256** + splitmix64        cuda/braid_knot.cu:56-90
 *   proposal     draw_freqs / split_unit / propose cuda/braid_knot.cu:111-166
 *   z grid       z_i = (i+1) pi / (T+1)            cuda/braid_knot.cu:309-320
 *   evaluation   a (sin(bz) cos f + cos(bz) sin f - sin f) / sin z + a2
 *                                                  cuda/braid_knot.cu:346-358
 *   wrap / delta torus_wrap, torus_delta           cuda/braid_knot.cu:168-178
 *   exclusion    Chebyshev per timestep            cuda/braid_knot.cu:359-372
 *   admission    in index order, each candidate checked against every
 *                earlier admission                 cuda/braid_knot.cu:433-462
 *   subpaths     join iff all contacts share one group id
 *                                                  cuda/braid_cuda.cu:390-467, 726-750
 *   cell index   floor((X+1)/cell), neighbours mod gw
 *                                                  cuda/braid_cuda.cu:700-702
 * plus the Philox candidate stream of the B200 packer (no reference
 * counterpart): Philox4x32-10 from Salmon et al., SC'11.
 *
 * Compiled with plain gcc (no -ffast-math, no FMA contraction) so the
 * arithmetic follows the C source operation by operation.
 */
#include "ug_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static const double kPi = 3.14159265358979323846;

/* ------------------------------------------------------------------ RNGs */

typedef struct {
    uint64_t s[4];
} xo_t;

static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static void xo_seed(xo_t* r, uint64_t seed) {
    for (int i = 0; i < 4; i++) {
        seed += 0x9E3779B97F4A7C15ULL;
        uint64_t z = seed;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        r->s[i] = z ^ (z >> 31);
    }
}

static uint64_t xo_next(xo_t* r) {
    uint64_t result = rotl64(r->s[1] * 5, 7) * 9;
    uint64_t t = r->s[1] << 17;
    r->s[2] ^= r->s[0];
    r->s[3] ^= r->s[1];
    r->s[1] ^= r->s[2];
    r->s[0] ^= r->s[3];
    r->s[2] ^= t;
    r->s[3] = rotl64(r->s[3], 45);
    return result;
}

static double xo_f64(xo_t* r) { return (double)(xo_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t xo_below(xo_t* r, uint32_t n) { return (uint32_t)(xo_next(r) % n); }
static int xo_flip(xo_t* r) { return (int)(xo_next(r) & 1ULL); }

void ora_xoshiro_stream(uint64_t seed, int32_t n, uint64_t* out) {
    xo_t r;
    xo_seed(&r, seed);
    for (int i = 0; i < n; i++) out[i] = xo_next(&r);
}

void ora_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; round++) {
        if (round) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* ------------------------------------------------------------ candidate */

typedef struct {
    int32_t b[3][ORA_MAX_F];
    double a[3][ORA_MAX_F];
    double f[3][ORA_MAX_F];
    double a2[3];
} cand_t;

static int modmax_of(int T) { return T - 1 > 2 ? T - 1 : 2; }

/* braid_knot.cu:111-166, draw for draw. */
static void propose_knot(const ora_model* m, uint64_t idx, cand_t* c) {
    xo_t r;
    xo_seed(&r, m->seed ^ (idx * 0x9E3779B97F4A7C15ULL + 0x1234567ULL));
    const uint32_t modmax = (uint32_t)modmax_of(m->T);
    const int nw = m->nw;
    double w[ORA_MAX_F];
    for (int ax = 0; ax < m->dim; ax++) {
        int32_t* out = c->b[ax];
        if ((uint32_t)nw == modmax) { /* full pool: identity + Fisher-Yates */
            for (int j = 0; j < nw; j++) out[j] = j + 2;
            for (int j = nw - 1; j > 0; j--) {
                int k = (int)xo_below(&r, (uint32_t)(j + 1));
                int tmp = out[j];
                out[j] = out[k];
                out[k] = tmp;
            }
        } else { /* rejection draws, 64 tries, no fallback (braid_knot.cu:134-145) */
            for (int j = 0; j < nw; j++) {
                int bnew = 0;
                int dup = 1;
                for (int guard = 0; dup && guard < 64; guard++) {
                    bnew = (int)xo_below(&r, modmax) + 2;
                    dup = 0;
                    for (int k = 0; k < j; k++)
                        if (out[k] == bnew) dup = 1;
                }
                out[j] = bnew;
            }
        }
        double sum = 0.0; /* exponential spacings (braid_knot.cu:98-107) */
        for (int j = 0; j < nw; j++) {
            w[j] = -log(1.0 - xo_f64(&r));
            sum += w[j];
        }
        for (int j = 0; j < nw; j++) w[j] /= sum;
        for (int j = 0; j < nw; j++) {
            double amp = w[j] / (double)out[j];
            if (xo_flip(&r)) amp = -amp;
            c->a[ax][j] = amp;
            c->f[ax][j] = (out[j] % 2 == 0) ? xo_f64(&r) * kPi : 0.0;
        }
        c->a2[ax] = m->pin ? 0.0 : (xo_f64(&r) * 2.0 - 1.0);
    }
}

/* Philox candidate stream of the B200 packer.  Key = seed, counter =
 * (idx_lo, idx_hi, axis<<16 | p, 0).  Block p >= 1 serves the frequency pair
 * (2p, 2p+1): words 0/1 -> exponential variates E = -log((r + 1/2) 2^-32),
 * word 2 -> even-b sign (bit 0) and phase f = (r >> 1) 2^-31 pi, word 3 ->
 * odd-b sign (bit 0).  Block 0 word 0 -> sin1 amplitude a2 = r 2^-31 - 1.
 * Weights w_b = E_b / sum_{b=2..F} E_b (ascending b), a_b = +-w_b / b. */
static void propose_philox(const ora_model* m, uint64_t idx, cand_t* c) {
    const int F = m->T;
    const uint32_t key[2] = {(uint32_t)m->seed, (uint32_t)(m->seed >> 32)};
    double E[ORA_MAX_F + 2];
    int sgn[ORA_MAX_F + 2];
    double ph[ORA_MAX_F + 2];
    for (int ax = 0; ax < m->dim; ax++) {
        uint32_t o[4];
        for (int p = 0; 2 * p <= F; p++) {
            const uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)(idx >> 32),
                                     ((uint32_t)ax << 16) | (uint32_t)p, 0u};
            ora_philox4x32_10(ctr, key, o);
            if (p == 0) {
                c->a2[ax] = m->pin ? 0.0 : (double)o[0] * (1.0 / 2147483648.0) - 1.0;
                continue;
            }
            const int be = 2 * p, bo = 2 * p + 1;
            E[be] = -log(((double)o[0] + 0.5) * (1.0 / 4294967296.0));
            sgn[be] = (int)(o[2] & 1u);
            ph[be] = (double)(o[2] >> 1) * (1.0 / 2147483648.0) * kPi;
            if (bo <= F) {
                E[bo] = -log(((double)o[1] + 0.5) * (1.0 / 4294967296.0));
                sgn[bo] = (int)(o[3] & 1u);
                ph[bo] = 0.0;
            }
        }
        double sum = 0.0;
        for (int b = 2; b <= F; b++) sum += E[b];
        for (int b = 2; b <= F; b++) {
            const int j = b - 2;
            const double wb = E[b] / sum;
            double amp = wb / (double)b;
            if (sgn[b]) amp = -amp;
            c->b[ax][j] = b;
            c->a[ax][j] = amp;
            c->f[ax][j] = ph[b];
        }
    }
}

static void propose(const ora_model* m, uint64_t idx, cand_t* c) {
    if (m->rng == ORA_RNG_KNOT)
        propose_knot(m, idx, c);
    else
        propose_philox(m, idx, c);
}

/* --------------------------------------------------------------- tables */

typedef struct {
    int T, F, dim, gw;
    double cell;     /* exclusion radius == grid cell width */
    int inclusive;   /* 1: |d| <= cell, 0: |d| < cell */
    int euclid;      /* L2 ball of radius cell (cuda/braid_cuda3d.cu:605-608) */
    double* z;
    double* sinz;
    double* invsinz;
    double* S; /* sin(b z_t)  [(F+1) * T] */
    double* C; /* cos(b z_t)  [(F+1) * T] */
    int* order;
} tabs_t;

static int tabs_init(const ora_model* m, tabs_t* tb) {
    const int T = m->T, F = m->T;
    tb->T = T;
    tb->F = F;
    tb->dim = m->dim;
    tb->euclid = m->euclid;
    if (m->excl == ORA_EXCL_REF) {
        tb->cell = 2.0 / T;
        tb->gw = T;
        tb->inclusive = 1;
    } else {
        tb->cell = 1.0 / F;
        tb->gw = 2 * F;
        tb->inclusive = 0;
    }
    tb->z = malloc(sizeof(double) * T);
    tb->sinz = malloc(sizeof(double) * T);
    tb->invsinz = malloc(sizeof(double) * T);
    tb->S = malloc(sizeof(double) * (size_t)(F + 1) * T);
    tb->C = malloc(sizeof(double) * (size_t)(F + 1) * T);
    tb->order = malloc(sizeof(int) * T);
    if (!tb->z || !tb->sinz || !tb->invsinz || !tb->S || !tb->C || !tb->order) return -1;
    for (int i = 0; i < T; i++) {
        if (m->zgrid == ORA_ZGRID_REF)
            tb->z[i] = (i + 1) * kPi / (T + 1);
        else
            tb->z[i] = (i + 0.5) * kPi / T;
        tb->sinz[i] = sin(tb->z[i]);
        tb->invsinz[i] = 1.0 / tb->sinz[i];
    }
    for (int b = 0; b <= F; b++)
        for (int t = 0; t < T; t++) {
            tb->S[(size_t)b * T + t] = sin(b * tb->z[t]);
            tb->C[(size_t)b * T + t] = cos(b * tb->z[t]);
        }
    /* endpoint-first visiting order (braid_cuda.cu:663-664): min(i, T-1-i)
     * ascending, ties by index.  Decisions do not depend on it. */
    for (int i = 0; i < T; i++) tb->order[i] = i;
    for (int i = 1; i < T; i++) {
        int v = tb->order[i], k = i;
        int kv = v < T - 1 - v ? v : T - 1 - v;
        while (k > 0) {
            int u = tb->order[k - 1];
            int ku = u < T - 1 - u ? u : T - 1 - u;
            if (ku <= kv) break;
            tb->order[k] = u;
            k--;
        }
        tb->order[k] = v;
    }
    return 0;
}

static void tabs_free(tabs_t* tb) {
    free(tb->z);
    free(tb->sinz);
    free(tb->invsinz);
    free(tb->S);
    free(tb->C);
    free(tb->order);
}

int ora_tables(const ora_model* m, double* z, double* invsinz, double* S, double* C) {
    tabs_t tb;
    if (tabs_init(m, &tb)) return -1;
    const int T = m->T;
    memcpy(z, tb.z, sizeof(double) * T);
    memcpy(invsinz, tb.invsinz, sizeof(double) * T);
    memcpy(S, tb.S, sizeof(double) * (size_t)(T + 1) * T);
    memcpy(C, tb.C, sizeof(double) * (size_t)(T + 1) * T);
    tabs_free(&tb);
    return 0;
}

static double torus_wrap(double x) { return x - 2.0 * floor((x + 1.0) * 0.5); }
static double torus_delta(double d) {
    if (d > 1.0) return d - 2.0;
    if (d < -1.0) return d + 2.0;
    return d;
}

/* Per-candidate evaluation state: trig of the phases, once per candidate. */
typedef struct {
    cand_t c;
    double cf[3][ORA_MAX_F], sf[3][ORA_MAX_F];
    double alpha[3][ORA_MAX_F + 1], beta[3][ORA_MAX_F + 1];
    int knot;
} ev_t;

static void ev_prepare(const ora_model* m, ev_t* e) {
    e->knot = m->rng == ORA_RNG_KNOT;
    const int F = m->T;
    for (int ax = 0; ax < m->dim; ax++) {
        for (int b = 0; b <= F; b++) e->alpha[ax][b] = e->beta[ax][b] = 0.0;
        for (int j = 0; j < m->nw; j++) {
            e->cf[ax][j] = cos(e->c.f[ax][j]);
            e->sf[ax][j] = sin(e->c.f[ax][j]);
            const int b = e->c.b[ax][j];
            e->alpha[ax][b] += e->c.a[ax][j] * e->cf[ax][j];
            e->beta[ax][b] += e->c.a[ax][j] * e->sf[ax][j];
        }
    }
}

/* Wrapped position of one axis at timestep t.  Knot mode follows the
 * reference host evaluation term for term (braid_knot.cu:346-358); the
 * Philox mode uses the packer's canonical sine-basis form
 *   X = wrap(a2 + invsinz_t * sum_{b=2..F} (alpha_b S_bt + beta_b (C_bt - 1))). */
static double ev_pos(const ora_model* m, const tabs_t* tb, const ev_t* e, int ax, int t) {
    const int T = tb->T;
    if (e->knot) {
        double wig = 0.0;
        for (int j = 0; j < m->nw; j++) {
            const int b = e->c.b[ax][j];
            wig += e->c.a[ax][j] * (tb->S[(size_t)b * T + t] * e->cf[ax][j] +
                                    tb->C[(size_t)b * T + t] * e->sf[ax][j] - e->sf[ax][j]);
        }
        return torus_wrap(wig * tb->invsinz[t] + e->c.a2[ax]);
    }
    double acc = 0.0;
    for (int b = 2; b <= tb->F; b++) {
        acc += e->alpha[ax][b] * tb->S[(size_t)b * T + t];
        acc += e->beta[ax][b] * (tb->C[(size_t)b * T + t] - 1.0);
    }
    return torus_wrap(acc * tb->invsinz[t] + e->c.a2[ax]);
}

int ora_candidate(const ora_model* m, uint64_t idx, int32_t* b, double* a, double* f, double* a2,
                  double* alpha, double* beta) {
    if (m->dim < 1 || m->dim > 3 || m->T < 4 || m->T > ORA_MAX_F || m->nw < 1 || m->nw > m->T - 1)
        return -1;
    ev_t* e = malloc(sizeof(ev_t));
    if (!e) return -1;
    propose(m, idx, &e->c);
    ev_prepare(m, e);
    for (int ax = 0; ax < m->dim; ax++) {
        for (int j = 0; j < m->nw; j++) {
            if (b) b[ax * m->nw + j] = e->c.b[ax][j];
            if (a) a[ax * m->nw + j] = e->c.a[ax][j];
            if (f) f[ax * m->nw + j] = e->c.f[ax][j];
        }
        if (a2) a2[ax] = e->c.a2[ax];
        for (int bb = 0; bb <= m->T; bb++) {
            if (alpha) alpha[ax * (m->T + 1) + bb] = e->alpha[ax][bb];
            if (beta) beta[ax * (m->T + 1) + bb] = e->beta[ax][bb];
        }
    }
    free(e);
    return 0;
}

int ora_positions(const ora_model* m, uint64_t idx, double* pos) {
    if (m->dim < 1 || m->dim > 3 || m->T < 4 || m->T > ORA_MAX_F || m->nw < 1 || m->nw > m->T - 1)
        return -1;
    tabs_t tb;
    if (tabs_init(m, &tb)) return -1;
    ev_t* e = malloc(sizeof(ev_t));
    if (!e) {
        tabs_free(&tb);
        return -1;
    }
    propose(m, idx, &e->c);
    ev_prepare(m, e);
    for (int ax = 0; ax < m->dim; ax++)
        for (int t = 0; t < m->T; t++) pos[ax * m->T + t] = ev_pos(m, &tb, e, ax, t);
    free(e);
    tabs_free(&tb);
    return 0;
}

/* --------------------------------------------------------------- packing */

/* Accepted-path store: wrapped positions [n][dim][T], group ids, and a
 * per-timestep cell hash (open addressing, key = t<<40 | cell) whose values
 * head singly linked chains through next[path*T + t]. */
typedef struct {
    int dim, T, gw;
    int64_t n, cap;
    double* pos;
    int32_t* gid;
    int32_t* next;
    int64_t* hkey;
    int32_t* hval;
    int64_t hcap, hn;
} store_t;

static uint64_t mix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

static int64_t* hslot(store_t* s, int64_t key) {
    uint64_t h = mix64((uint64_t)key) & (uint64_t)(s->hcap - 1);
    while (s->hkey[h] != -1 && s->hkey[h] != key) h = (h + 1) & (uint64_t)(s->hcap - 1);
    return &s->hkey[h];
}

static int32_t hget(const store_t* s, int64_t key) {
    uint64_t h = mix64((uint64_t)key) & (uint64_t)(s->hcap - 1);
    while (s->hkey[h] != -1) {
        if (s->hkey[h] == key) return s->hval[h];
        h = (h + 1) & (uint64_t)(s->hcap - 1);
    }
    return -1;
}

static int hrehash(store_t* s, int64_t ncap) {
    int64_t* ok = s->hkey;
    int32_t* ov = s->hval;
    int64_t oc = s->hcap;
    s->hkey = malloc(sizeof(int64_t) * ncap);
    s->hval = malloc(sizeof(int32_t) * ncap);
    if (!s->hkey || !s->hval) return -1;
    for (int64_t i = 0; i < ncap; i++) s->hkey[i] = -1;
    s->hcap = ncap;
    for (int64_t i = 0; i < oc; i++)
        if (ok[i] != -1) {
            int64_t* k = hslot(s, ok[i]);
            *k = ok[i];
            s->hval[k - s->hkey] = ov[i];
        }
    free(ok);
    free(ov);
    return 0;
}

static int store_init(store_t* s, int dim, int T, int gw) {
    memset(s, 0, sizeof(*s));
    s->dim = dim;
    s->T = T;
    s->gw = gw;
    s->cap = 1024;
    s->pos = malloc(sizeof(double) * s->cap * dim * T);
    s->gid = malloc(sizeof(int32_t) * s->cap);
    s->next = malloc(sizeof(int32_t) * s->cap * T);
    s->hcap = 1 << 16;
    s->hkey = malloc(sizeof(int64_t) * s->hcap);
    s->hval = malloc(sizeof(int32_t) * s->hcap);
    if (!s->pos || !s->gid || !s->next || !s->hkey || !s->hval) return -1;
    for (int64_t i = 0; i < s->hcap; i++) s->hkey[i] = -1;
    return 0;
}

static void store_free(store_t* s) {
    free(s->pos);
    free(s->gid);
    free(s->next);
    free(s->hkey);
    free(s->hval);
}

static int cell_of(double X, double cell, int gw) {
    int c = (int)floor((X + 1.0) / cell);
    if (c >= gw) c = gw - 1; /* X -> 1^- rounding; the true cell is gw-1 */
    if (c < 0) c = 0;
    return c;
}

static int64_t cell_key(int t, const int* c, int dim, int gw) {
    int64_t lin = 0;
    for (int ax = 0; ax < dim; ax++) lin = lin * gw + c[ax];
    return ((int64_t)t << 40) | lin;
}

static int store_add(store_t* s, const double* P /* [dim][T] */, int32_t gid, double cell, int64_t* new_cells) {
    if (s->n == s->cap) {
        int64_t nc = s->cap * 2;
        double* np = realloc(s->pos, sizeof(double) * nc * s->dim * s->T);
        int32_t* ng = realloc(s->gid, sizeof(int32_t) * nc);
        int32_t* nn = realloc(s->next, sizeof(int32_t) * nc * s->T);
        if (!np || !ng || !nn) return -1;
        s->pos = np;
        s->gid = ng;
        s->next = nn;
        s->cap = nc;
    }
    const int64_t p = s->n;
    memcpy(&s->pos[p * s->dim * s->T], P, sizeof(double) * s->dim * s->T);
    s->gid[p] = gid;
    if ((s->hn + s->T) * 2 > s->hcap)
        if (hrehash(s, s->hcap * 2)) return -1;
    for (int t = 0; t < s->T; t++) {
        int c[3];
        for (int ax = 0; ax < s->dim; ax++) c[ax] = cell_of(P[ax * s->T + t], cell, s->gw);
        const int64_t key = cell_key(t, c, s->dim, s->gw);
        int64_t* k = hslot(s, key);
        if (*k == -1) {
            *k = key;
            s->hval[k - s->hkey] = -1;
            s->hn++;
            ++*new_cells;
        }
        s->next[p * s->T + t] = s->hval[k - s->hkey];
        s->hval[k - s->hkey] = (int32_t)p;
    }
    s->n++;
    return 0;
}

static int hit1(double d, double cell, int inclusive) {
    const double ad = fabs(d);
    return inclusive ? ad <= cell : ad < cell;
}

/* Exclusion test of two points (axis ax of P at P[ax * ps], of Q at Q[ax * qs]):
 * the Chebyshev cube of half-width cell, or with euclid the L2 ball
 * dX*dX + dY*dY + dW*dW <= cell*cell (cuda/braid_cuda3d.cu:605-608, summed
 * in that order; this file is built without floating-point contraction). */
static int pair_hit(const tabs_t* tb, int dim, const double* P, int64_t ps, const double* Q, int64_t qs) {
    if (!tb->euclid) {
        for (int ax = 0; ax < dim; ax++)
            if (!hit1(torus_delta(P[ax * ps] - Q[ax * qs]), tb->cell, tb->inclusive)) return 0;
        return 1;
    }
    double s = 0.0;
    for (int ax = 0; ax < dim; ax++) {
        const double d = torus_delta(P[ax * ps] - Q[ax * qs]);
        s = s + d * d;
    }
    const double r2 = tb->cell * tb->cell;
    return tb->inclusive ? s <= r2 : s < r2;
}

/* Contacts of position vector Pt (one timestep) with stored paths at t.
 * Unique mode returns 1 on the first contact.  Group mode collects ids into
 * *g0 and returns 1 as soon as a second distinct id appears. */
static int contacts_at(const store_t* s, const tabs_t* tb, int t, const double* Pt, int group,
                       int32_t* g0) {
    int c[3];
    for (int ax = 0; ax < s->dim; ax++) c[ax] = cell_of(Pt[ax], tb->cell, tb->gw);
    int nb = 1;
    for (int ax = 0; ax < s->dim; ax++) nb *= 3;
    for (int k = 0; k < nb; k++) {
        int cc[3], r = k;
        for (int ax = s->dim - 1; ax >= 0; ax--) {
            const int dd = r % 3 - 1;
            r /= 3;
            cc[ax] = (c[ax] + dd + tb->gw) % tb->gw;
        }
        /* gw == 2 or 3 would visit a cell twice; harmless for the predicate */
        int32_t p = hget(s, cell_key(t, cc, s->dim, tb->gw));
        while (p >= 0) {
            const double* Q = &s->pos[(int64_t)p * s->dim * s->T];
            const int hit = pair_hit(tb, s->dim, Pt, 1, Q + t, s->T);
            if (hit) {
                if (!group) return 1;
                if (*g0 == -1)
                    *g0 = s->gid[p];
                else if (*g0 != s->gid[p])
                    return 1;
            }
            p = s->next[(int64_t)p * s->T + t];
        }
    }
    return 0;
}

/* 1+1D crossing rule: the minimum-image separation changes sign between
 * consecutive timesteps while |d_t| + |d_t+1| < 1 (a crossing through 0, not
 * an antipodal flip through +-1).  No reference counterpart. */
static int crosses(const double* P, const double* Q, int T) {
    double d0 = torus_delta(P[0] - Q[0]);
    for (int t = 0; t + 1 < T; t++) {
        const double d1 = torus_delta(P[t + 1] - Q[t + 1]);
        if (((d0 < 0.0) != (d1 < 0.0)) && fabs(d0) + fabs(d1) < 1.0) return 1;
        d0 = d1;
    }
    return 0;
}

typedef struct {
    const ora_model* m;
    const tabs_t* tb;
    ev_t ev;
    double P[3 * ORA_MAX_F];
    int have[ORA_MAX_F];
} cand_eval_t;

static void ce_start(cand_eval_t* ce, uint64_t idx) {
    propose(ce->m, idx, &ce->ev.c);
    ev_prepare(ce->m, &ce->ev);
    for (int t = 0; t < ce->m->T; t++) ce->have[t] = 0;
}

static void ce_at(cand_eval_t* ce, int t, double* Pt) {
    const int T = ce->m->T;
    if (!ce->have[t]) {
        for (int ax = 0; ax < ce->m->dim; ax++)
            ce->P[ax * T + t] = ev_pos(ce->m, ce->tb, &ce->ev, ax, t);
        ce->have[t] = 1;
    }
    for (int ax = 0; ax < ce->m->dim; ax++) Pt[ax] = ce->P[ax * T + t];
}

static void ce_all(cand_eval_t* ce) {
    double Pt[3];
    for (int t = 0; t < ce->m->T; t++) ce_at(ce, t, Pt);
}

/* Test the current candidate against stored paths with index in [lo, hi).
 * Returns: unique mode -> 1 collides / 0 free.
 * Group mode -> sets *g (-1 none, >=0 the single group) and returns 1 when
 * two distinct groups are touched. */
static int ce_test(cand_eval_t* ce, const store_t* s, int group, int32_t* g) {
    const ora_model* m = ce->m;
    const int T = m->T;
    *g = -1;
    if (m->dim == 1 && m->cross1d) {
        ce_all(ce);
        for (int64_t p = 0; p < s->n; p++) {
            const double* Q = &s->pos[p * T];
            int hit = crosses(ce->P, Q, T);
            for (int t = 0; t < T && !hit; t++)
                hit = hit1(torus_delta(ce->P[t] - Q[t]), ce->tb->cell, ce->tb->inclusive);
            if (hit) {
                if (!group) return 1;
                if (*g == -1)
                    *g = s->gid[p];
                else if (*g != s->gid[p])
                    return 1;
            }
        }
        return 0;
    }
    double Pt[3];
    for (int oi = 0; oi < T; oi++) {
        const int t = ce->tb->order[oi];
        ce_at(ce, t, Pt);
        if (contacts_at(s, ce->tb, t, Pt, group, g)) return 1;
    }
    return 0;
}

static int record(ora_result* res, int64_t idx, int32_t gid) {
    if (res->n_acc >= res->cap) return -2;
    res->acc_idx[res->n_acc] = idx;
    if (res->gid) res->gid[res->n_acc] = gid;
    res->n_acc++;
    return 0;
}

/* ---- windowed stops (the --until-accept-rate window of braid_cuda.cu:585-590,
 * 931-943 and the phase-2 new-volume window of braid_cuda.cu:953-1037).  The
 * reference keeps a deque of its rounds' (batch, admitted) pairs covering at
 * least win_target = clamp(30 / threshold, 2e7, 5e9) attempts and stops when
 * the window's rate falls below the threshold after 1e6 attempts.  Its rounds
 * are its own adaptive batches; here the window is made of 32 buckets of
 * q = win_target / 32 candidates aligned at the phase start, so the stop point
 * is a function of the candidate stream alone: at every bucket boundary (in
 * phase-relative candidates) the last 32 buckets are summed, and the phase
 * ends there when 32 buckets exist, more than 1e6 candidates are decided and
 * sum / (32 q) < threshold.  The packer evaluates the same rule at the same
 * boundaries (its rounds never straddle one). */
typedef struct {
    double thr;
    int64_t q;
    int64_t ring[32];
    int64_t nb, sum, cur;
} win_t;

static void win_init(win_t* w, double thr) {
    memset(w, 0, sizeof(*w));
    w->thr = thr;
    if (thr > 0) {
        double t = 30.0 / thr;
        if (t < 2e7) t = 2e7;
        if (t > 5e9) t = 5e9;
        const int64_t W = (int64_t)t;
        w->q = W / 32 > 0 ? W / 32 : 1;
    }
}

/* candidates from phase position in_phase to the next bucket boundary */
static int64_t win_room(const win_t* w, int64_t in_phase) {
    return w->q ? w->q - in_phase % w->q : INT64_MAX;
}

/* Called once candidates [0, in_phase) of the phase are decided; returns 1
 * when the phase stops at in_phase. */
static int win_close(win_t* w, int64_t in_phase) {
    if (!w->q || in_phase <= 0 || in_phase % w->q) return 0;
    const int slot = (int)(w->nb & 31);
    if (w->nb >= 32) w->sum -= w->ring[slot];
    w->ring[slot] = w->cur;
    w->sum += w->cur;
    w->cur = 0;
    w->nb++;
    return w->nb >= 32 && in_phase > 1000000 && (double)w->sum / (double)(32 * w->q) < w->thr;
}

/* ---- admission rules.  mode 0: unique packing (any contact rejects);
 * mode 1: unique-group (no contact founds a group labelled by its slot, one
 * group joins it, two or more reject); mode 2: subpath phase (exactly one group
 * joins, braid_cuda.cu:726-750).  The first test against the committed packing
 * is also the threaded prefilter: a rejection there is final because the
 * packing only grows and group labels never change. */
static int decide(cand_eval_t* ce, const store_t* s, int mode, int32_t* gid, int* founded) {
    int32_t g;
    if (mode == 0) {
        if (ce_test(ce, s, 0, &g)) return 0;
        *gid = (int32_t)s->n;
        *founded = 1;
        return 1;
    }
    if (ce_test(ce, s, 1, &g)) return 0;
    if (g < 0) {
        if (mode == 2) return 0;
        *gid = (int32_t)s->n;
        *founded = 1;
        return 1;
    }
    *gid = g;
    *founded = 0;
    return 1;
}

/* ---- threaded form: parallel prefilter of a batch against the committed
 * packing, then the serial in-order decision of the survivors against the
 * packing including the batch's earlier admissions (the scheme of
 * braid_knot.cu:401-469 with CPU threads in place of the kernel; the decisions
 * are those of the sequential loop). */
typedef struct {
    const ora_model* m;
    const tabs_t* tb;
    const store_t* s;
    int64_t base, count;
    uint8_t* surv;
    int tid, nth, mode;
} mt_job_t;

static void* mt_worker(void* arg) {
    mt_job_t* j = (mt_job_t*)arg;
    cand_eval_t* ce = malloc(sizeof(cand_eval_t));
    if (!ce) return (void*)1;
    ce->m = j->m;
    ce->tb = j->tb;
    const int64_t per = (j->count + j->nth - 1) / j->nth;
    const int64_t lo = (int64_t)j->tid * per;
    const int64_t hi = lo + per < j->count ? lo + per : j->count;
    for (int64_t i = lo; i < hi; i++) {
        int32_t g;
        ce_start(ce, (uint64_t)(j->base + i));
        j->surv[i] = (uint8_t)!ce_test(ce, j->s, j->mode != 0, &g);
    }
    free(ce);
    return NULL;
}

/* One phase over candidates [start, start + budget): admissions in index order
 * under rule `mode`, stopped early by max_n (phase-1 uniques) or a window. */
static int run_phase(const ora_model* m, const ora_run* run, const tabs_t* tb, store_t* s, ora_result* res,
                     int mode, int64_t start, int64_t budget, int64_t max_n, double acc_thr, double fill_thr,
                     int64_t* end_out) {
    const int nth = run->nthreads > 1 ? run->nthreads : 1;
    const int64_t B = nth > 1 ? (run->round > 0 ? run->round : 65536) : 1;
    uint8_t* surv = nth > 1 ? malloc((size_t)B) : NULL;
    pthread_t* th = malloc(sizeof(pthread_t) * nth);
    mt_job_t* jobs = malloc(sizeof(mt_job_t) * nth);
    cand_eval_t* ce = malloc(sizeof(cand_eval_t));
    int rc = 0;
    if ((nth > 1 && !surv) || !th || !jobs || !ce) {
        rc = -1;
        goto done;
    }
    ce->m = m;
    ce->tb = tb;
    win_t wa, wf;
    win_init(&wa, acc_thr);
    win_init(&wf, fill_thr);
    const int64_t end = start + budget;
    int64_t idx = start;
    while (idx < end && !(max_n && res->n_unique >= max_n)) {
        const int64_t in0 = idx - start;
        int64_t cnt = end - idx < B ? end - idx : B;
        if (win_room(&wa, in0) < cnt) cnt = win_room(&wa, in0);
        if (win_room(&wf, in0) < cnt) cnt = win_room(&wf, in0);
        if (nth > 1) {
            for (int k = 0; k < nth; k++) {
                jobs[k] = (mt_job_t){m, tb, s, idx, cnt, surv, k, nth, mode};
                pthread_create(&th[k], NULL, mt_worker, &jobs[k]);
            }
            for (int k = 0; k < nth; k++) pthread_join(th[k], NULL);
        }
        int64_t consumed = cnt, adm = 0, newc = 0;
        for (int64_t i = 0; i < cnt; i++) {
            if (surv && !surv[i]) continue;
            int32_t gid;
            int founded;
            ce_start(ce, (uint64_t)(idx + i));
            if (!decide(ce, s, mode, &gid, &founded)) continue;
            ce_all(ce);
            if (store_add(s, ce->P, gid, tb->cell, &newc) || record(res, idx + i, gid)) {
                rc = -2;
                goto done;
            }
            adm++;
            if (founded)
                res->n_unique++;
            else
                res->n_sub++;
            if (max_n && res->n_unique >= max_n) {
                consumed = i + 1;
                break;
            }
        }
        idx += consumed;
        wa.cur += adm;
        wf.cur += newc;
        const int sa = win_close(&wa, idx - start);
        const int sf = win_close(&wf, idx - start);
        if (sa || sf) break;
    }
    *end_out = idx;
done:
    free(surv);
    free(th);
    free(jobs);
    free(ce);
    return rc;
}

int ora_pack(const ora_model* m, const ora_run* run, ora_result* res) {
    if (m->dim < 1 || m->dim > 3 || m->T < 4 || m->T > ORA_MAX_F || m->nw < 1 || m->nw > m->T - 1)
        return -1;
    if (m->rng == ORA_RNG_PHILOX && m->nw != m->T - 1) return -1;
    tabs_t tb;
    if (tabs_init(m, &tb)) return -1;
    store_t s;
    if (store_init(&s, m->dim, m->T, tb.gw)) return -1;
    res->n_acc = res->n_unique = res->n_sub = res->attempts = res->phase1_end = 0;
    int64_t idx = 0;
    /* phase 1 (or the single unique-group phase) */
    int rc = run_phase(m, run, &tb, &s, res, run->group_mode == ORA_GROUP_UNIQUE ? 1 : 0, 0, run->attempts,
                       run->max_n, run->accept_rate, 0.0, &idx);
    res->phase1_end = idx;
    /* phase 2: subpaths (the candidate stream continues after phase 1) */
    if (!rc && run->group_mode == ORA_GROUP_SUBPATH)
        rc = run_phase(m, run, &tb, &s, res, 2, idx, run->sub_attempts > 0 ? run->sub_attempts : run->attempts, 0,
                       run->sub_accept_rate, run->sub_fill_rate, &idx);
    res->attempts = idx;
    store_free(&s);
    tabs_free(&tb);
    return rc;
}
