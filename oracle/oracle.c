/*
 * CPU oracle for the fixed-dt spiking hot path -- TEST INFRASTRUCTURE ONLY
 * (see oracle.h for what it restates and who may call it).
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off: every float operation is
 * rounded on its own, as the CUDA path's __fmul_rn/__fadd_rn are).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 1;

/* Threads of or_run (1: the sequential restatement; more: an OpenMP build,
 * the CPU baseline's "all host threads" -- integer sums make the result the
 * same). */
int or_set_threads(int n) {
#ifdef _OPENMP
    g_threads = n > 0 ? n : omp_get_max_threads();
#else
    (void)n;
    g_threads = 1;
#endif
    return g_threads;
}

/* ---------------------------------------------------------------- Philox */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies, the key
 * bumped by the Weyl constants between rounds. Triton's tl.randint, which the
 * reference's random lowering calls (naer2/transpiler/transformers/
 * random_lowering_transformer.py:74-86), is this generator with counter
 * (offset, 0, 0, 0) and key (seed low, seed high). */
void or_philox4x32_10(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]) {
    uint32_t c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
    uint32_t k0 = k[0], k1 = k[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* The population's draw for neuron j at step n, stream `purpose`
 * (0: external Poisson drive, 1: Poisson source): the first Philox word of
 * counter (j, n low, n high, purpose) under the population's seed. */
static uint32_t draw(const or_pop *p, int32_t j, int64_t n, uint32_t purpose) {
    uint32_t c[4] = {(uint32_t)j, (uint32_t)(uint64_t)n, (uint32_t)((uint64_t)n >> 32), purpose};
    uint32_t k[2] = {(uint32_t)p->seed, (uint32_t)(p->seed >> 32)};
    uint32_t out[4];
    or_philox4x32_10(c, k, out);
    return out[0];
}

/* Poisson count by inversion: the number of table entries the uniform word
 * is at or above (table[k] = floor(2^32 * P(X <= k)), built on the host in
 * fp64 and shared with the CUDA path). */
static int32_t poisson_count(const uint32_t *table, int32_t len, uint32_t u) {
    int32_t k = 0;
    while (k < len - 1 && u >= table[k]) ++k;
    return k;
}

int64_t or_wfx(float w, int32_t shift) {
    float scaled = ldexpf(w, shift); /* exact: a power-of-two scale */
    return (int64_t)llrintf(scaled); /* round to nearest, ties to even */
}

/* float(sum * 2^-shift): the int64 rounded to float once, then an exact scale. */
static float fx_to_float(int64_t acc, int32_t shift) {
    float f = (float)acc;
    return ldexpf(f, -shift);
}

/* ---------------------------------------------------------------- models */

/* LIF with delta synapses, time-driven (tools/brunel_reference.py:36-42):
 *   p[0] decay = fp32(exp(-dt/tau)), p[1] theta, p[2] V_reset.
 *   input = this step's slot (+ external Poisson events, in the same fixed-
 *   point sum); refractory (ref > 0): V kept, input dropped, ref counts down;
 *   else V = V * decay + input, fire at V >= theta, reset to V_reset,
 *   ref = ref_steps (round(t_ref / dt): brunel_reference.py's
 *   `t > ref_until` test leaves a neuron inactive for exactly that many steps). */
static int lif_delta(or_pop *p, int32_t j, float input) {
    if (p->ref[j] > 0) {
        p->ref[j] -= 1;
        return 0;
    }
    float v = p->v[j] * p->p[0];
    v = v + input;
    int fire = v >= p->p[1];
    if (fire) {
        v = p->p[2];
        p->ref[j] = p->ref_steps;
    }
    p->v[j] = v;
    return fire;
}

/* PD14 LIF with exponential current synapses, exact propagators at fixed dt
 * (test/networks/PD14/neuron.py:166-186, test/fused_reference.py:86-103):
 *   p[0] P_V, p[1] P_I, p[2] P_VI, p[3] V_rest, p[4] V_thresh, p[5] V_reset.
 *   current += input (receive, before update); refractory: V = V_reset, else
 *   V = V_rest + P_V (V - V_rest) + P_VI current; current *= P_I; fire at
 *   V > V_thresh with reset and ref = ref_steps (round(t_ref / dt) - 1: the
 *   hook's `time < t_ref_end` clamps that many steps after the spike). */
static int pd14(or_pop *p, int32_t j, float input) {
    float cur = p->i[j] + input;
    float v;
    if (p->ref[j] > 0) {
        p->ref[j] -= 1;
        v = p->p[5];
    } else {
        float dv = p->v[j] - p->p[3];
        float a = p->p[0] * dv;
        float b = p->p[3] + a;
        float c = p->p[2] * cur;
        v = b + c;
    }
    cur = p->p[1] * cur;
    int fire = v > p->p[4];
    if (fire) {
        v = p->p[5];
        p->ref[j] = p->ref_steps;
    }
    p->v[j] = v;
    p->i[j] = cur;
    return fire;
}

/* ---------------------------------------------------------------- the step loop */

/* One neuron's intake, update and send at step n; returns its spike (or -1 for a bad description). */
static int neuron_step(or_pop *p, int32_t j, int64_t n, int64_t *slot) {
    if (p->model == OR_MODEL_POISSON_SOURCE) return draw(p, j, n, 1u) < p->fire_threshold;
    int64_t a = slot ? slot[j] : 0;
    if (slot) slot[j] = 0;
    if (p->ext_counts) {
        if (n < p->ext_step0 || n >= p->ext_step0 + p->ext_steps) return -1;
        a += (int64_t)p->ext_counts[(size_t)(n - p->ext_step0) * (size_t)p->n + (size_t)j] * p->ext_wfx;
    } else if (p->ext_table && p->ext_len > 0) {
        a += (int64_t)poisson_count(p->ext_table, p->ext_len, draw(p, j, n, 0u)) * p->ext_wfx;
    }
    float input = fx_to_float(a, p->shift);
    if (p->model == OR_MODEL_LIF_DELTA) return lif_delta(p, j, input);
    if (p->model == OR_MODEL_PD14) return pd14(p, j, input);
    return -1;
}

/* A run of at most RUN links of one spike's outgoing row in one connection: the unit of the parallel
 * delivery (the sums are exact integers, so the units may run in any order). */
#define RUN 512
typedef struct {
    int32_t conn, first, end;
} or_unit;

int or_run(or_pop *pops, int32_t n_pops, const or_conn *conns, int32_t n_conns,
           int64_t step0, int64_t n_steps, uint64_t *events) {
    for (int32_t c = 0; c < n_conns; ++c) {
        if (conns[c].src < 0 || conns[c].src >= n_pops || conns[c].tgt < 0 || conns[c].tgt >= n_pops)
            return -1;
    }
    if (n_pops < 0 || n_conns < 0) return -1;
    int32_t total = 0, total_words = 0;
    for (int32_t q = 0; q < n_pops; ++q) {
        if (pops[q].n < 0 || (pops[q].acc_depth & (pops[q].acc_depth - 1)) != 0) return -1;
        total += pops[q].n;
        total_words += (pops[q].n + 31) / 32;
    }
    int32_t *spk = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total > 0 ? total : 1));
    int32_t *first = (int32_t *)calloc((size_t)n_pops + 1, sizeof(int32_t));
    int32_t *count = (int32_t *)calloc((size_t)n_pops + 1, sizeof(int32_t));
    /* per population its first word in the step's flat word list (every population's words in one loop) */
    int32_t *wfirst = (int32_t *)calloc((size_t)n_pops + 1, sizeof(int32_t));
    int32_t *wpop = (int32_t *)malloc(sizeof(int32_t) * (size_t)(total_words > 0 ? total_words : 1));
    uint32_t *mark = (uint32_t *)calloc((size_t)(total_words > 0 ? total_words : 1), sizeof(uint32_t));
    int64_t *wfx_const = (int64_t *)calloc((size_t)n_conns + 1, sizeof(int64_t));
    size_t cap = 1024;
    or_unit *units = (or_unit *)malloc(sizeof(or_unit) * cap);
    if (!spk || !first || !count || !wfirst || !wpop || !mark || !wfx_const || !units) {
        free(spk); free(first); free(count); free(wfirst); free(wpop); free(mark); free(wfx_const); free(units);
        return -3;
    }
    for (int32_t q = 0; q < n_pops; ++q) {
        first[q + 1] = first[q] + pops[q].n;
        wfirst[q + 1] = wfirst[q] + (pops[q].n + 31) / 32;
        for (int32_t w = wfirst[q]; w < wfirst[q + 1]; ++w) wpop[w] = q;
    }
    for (int32_t c = 0; c < n_conns; ++c) wfx_const[c] = or_wfx(conns[c].weight, pops[conns[c].tgt].shift);
    uint64_t ev = 0;
    int rc = 0;

    for (int64_t s = 0; s < n_steps && rc == 0; ++s) {
        int64_t n = step0 + s;
        /* update every neuron of every population from its due arrival slot (neurons are independent); one word
         * of 32 neurons per iteration: the raster word and the spike marks are the iteration's own */
        int bad = 0;
#pragma omp parallel for schedule(static) num_threads(g_threads) reduction(|:bad)
        for (int32_t gw = 0; gw < total_words; ++gw) {
            const int32_t q = wpop[gw], w = gw - wfirst[q];
            or_pop *p = &pops[q];
            int64_t *slot = p->acc ? p->acc + (size_t)(n & (p->acc_depth - 1)) * (size_t)p->n : NULL;
            uint32_t bits = 0;
            int32_t j1 = (w + 1) * 32 < p->n ? (w + 1) * 32 : p->n;
            for (int32_t j = w * 32; j < j1; ++j) {
                int fire = neuron_step(p, j, n, slot);
                if (fire < 0) { bad = 1; break; }
                if (fire) bits |= 1u << (j & 31);
            }
            mark[gw] = bits;
            if (p->raster && n >= p->raster_step0 && n < p->raster_step0 + p->raster_steps)
                p->raster[(size_t)(n - p->raster_step0) * (size_t)((p->n + 31) / 32) + (size_t)w] = bits;
        }
        if (bad) { rc = -4; break; }
        /* the spikes of this step, per population in index order */
        for (int32_t q = 0; q < n_pops; ++q) {
            count[q] = 0;
            for (int32_t gw = wfirst[q]; gw < wfirst[q + 1]; ++gw) {
                uint32_t bits = mark[gw];
                while (bits) {
                    int b = __builtin_ctz(bits);
                    bits &= bits - 1;
                    spk[first[q] + count[q]++] = (gw - wfirst[q]) * 32 + b;
                }
            }
        }
        /* the step's deliveries as runs of links: every spike's row in every outgoing connection */
        size_t nu = 0;
        for (int32_t c = 0; c < n_conns; ++c) {
            const or_conn *cn = &conns[c];
            for (int32_t k = 0; k < count[cn->src]; ++k) {
                int32_t s_id = spk[first[cn->src] + k];
                for (int32_t l = cn->ptr[s_id]; l < cn->ptr[s_id + 1]; l += RUN) {
                    if (nu == cap) {
                        or_unit *grown = (or_unit *)realloc(units, sizeof(or_unit) * cap * 2);
                        if (!grown) { rc = -3; break; }
                        units = grown;
                        cap *= 2;
                    }
                    int32_t e = cn->ptr[s_id + 1] - l > RUN ? l + RUN : cn->ptr[s_id + 1];
                    units[nu].conn = c;
                    units[nu].first = l;
                    units[nu].end = e;
                    ++nu;
                }
                if (rc) break;
            }
            if (rc) break;
        }
        if (rc) break;
        /* deliver: exact integer adds into the arrival slots, any order */
        uint64_t ev_s = 0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(g_threads) reduction(|:bad) reduction(+:ev_s)
        for (size_t u = 0; u < nu; ++u) {
            const or_conn *cn = &conns[units[u].conn];
            or_pop *tgt = &pops[cn->tgt];
            for (int32_t l = units[u].first; l < units[u].end; ++l) {
                uint32_t rec = cn->link[l];
                int32_t d = (int32_t)(rec >> 24), t = (int32_t)(rec & 0xFFFFFFu);
                if (d < 1 || d >= tgt->acc_depth || t >= tgt->n || !tgt->acc) { bad = 1; break; }
                int64_t wfx = cn->w ? or_wfx(cn->w[l], tgt->shift) : wfx_const[units[u].conn];
                int64_t *cell = &tgt->acc[(size_t)((n + d) & (tgt->acc_depth - 1)) * (size_t)tgt->n + (size_t)t];
                if (g_threads > 1) __atomic_fetch_add(cell, wfx, __ATOMIC_RELAXED);
                else *cell += wfx;
                ++ev_s;
            }
        }
        ev += ev_s;
        if (bad) rc = -2;
    }
    if (events) *events += ev;
    free(spk); free(first); free(count); free(wfirst); free(wpop); free(mark); free(wfx_const); free(units);
    return rc;
}

/* External counts of n neurons for steps [step0, step0 + n_steps) as the
 * step loop draws them (counter (j, n, 0), table inversion): out[steps][n]. */
void or_poisson_counts(const uint32_t *table, int32_t len, uint64_t seed, int64_t step0, int64_t n_steps,
                       int32_t n, int32_t *out) {
    or_pop p;
    memset(&p, 0, sizeof(p));
    p.seed = seed;
    for (int64_t s = 0; s < n_steps; ++s)
        for (int32_t j = 0; j < n; ++j)
            out[(size_t)s * (size_t)n + (size_t)j] = poisson_count(table, len, draw(&p, j, step0 + s, 0u));
}
