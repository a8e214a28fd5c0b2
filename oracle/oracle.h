/*
 * CPU oracle for the fixed-dt spiking hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * Nothing in the product links, imports or calls this code. Only tests/, the
 * smoke check in __graft_entry__.py and the CPU-baseline leg of bench.py use
 * it, and only as the checker (or as the timed CPU baseline), never as the
 * thing measured or shipped.
 *
 * It restates, in plain sequential C, the arithmetic of the reference's
 * time-driven paths:
 *   - the Brunel LIF step loop of tools/brunel_reference.py:34-48
 *     (input = delay-buffer slot + J * Poisson count; refractory neurons keep V;
 *     V = V * decay + input; fire at V >= theta; reset; refractory period);
 *   - the PD14 neuron hooks of test/networks/PD14/neuron.py:166-186 as the
 *     hand-written kernel test/fused_reference.py:86-103 runs them (receive adds
 *     the delivered weights to the current, then the exact propagator update,
 *     then the threshold test V > V_thresh with reset and refractory clamp);
 *   - the per-link arrival slot of test/test_fused_gpu.py:105-120
 *     (k = emission step + delay in steps, integer arithmetic here);
 *   - Philox4x32-10 (Salmon et al., SC'11), the generator behind the
 *     reference's tl.rand (naer2/transpiler/templates/fused.py:231-233),
 *     checked against the published known-answer vectors and Triton's own
 *     implementation by tests/test_oracle.py.
 *
 * Semantics shared with the CUDA path (and pinned by tests/golden/):
 *   - all synaptic input of a step is summed exactly in int64 fixed point
 *     (weight * 2^shift rounded to nearest-even, shift per target
 *     population) and converted to float once: the sum does not depend on
 *     the order of the additions;
 *   - a refractory period is an integer step counter.
 */
#ifndef NAER2_ORACLE_H
#define NAER2_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_MODEL_LIF_DELTA = 1, OR_MODEL_PD14 = 2, OR_MODEL_POISSON_SOURCE = 3 };

typedef struct {
    int32_t model;
    int32_t n;
    int32_t acc_depth;      /* power of two > the largest incoming delay in steps */
    int32_t shift;          /* fixed-point exponent of the input sum */
    int32_t ref_steps;      /* refractory steps set when a neuron fires */
    uint32_t fire_threshold;/* POISSON_SOURCE: fire when the uniform draw is below this */
    uint64_t seed;          /* Philox key of this population */
    float p[8];             /* model constants (see oracle.c) */
    int64_t ext_wfx;        /* fixed-point weight of one external Poisson event */
    const uint32_t *ext_table; /* inverse-CDF table of the external Poisson count, or NULL */
    int32_t ext_len;
    const int32_t *ext_counts; /* or given counts, [steps][n] from step ext_step0 (golden inputs) */
    int64_t ext_step0;
    int64_t ext_steps;
    float *v;               /* state: membrane potential */
    float *i;               /* state: synaptic current (PD14) */
    int32_t *ref;           /* state: refractory steps left */
    int64_t *acc;           /* [acc_depth][n] arrival-slot sums (fixed point) */
    uint32_t *raster;       /* [raster_steps][ceil(n/32)] spike bits, or NULL */
    int64_t raster_step0;   /* raster row 0 is this step */
    int64_t raster_steps;
} or_pop;

typedef struct {
    int32_t src, tgt;
    const int32_t *ptr;     /* [n_src + 1] outgoing CSR row offsets */
    const uint32_t *link;   /* (delay_steps << 24) | target */
    const float *w;         /* per-link weight, or NULL: `weight` for every link */
    float weight;
} or_conn;

/* Threads of or_run: 1 (default) the sequential restatement; n > 1 (or 0:
 * all) an OpenMP build's parallel one -- the same results. Returns the count. */
int or_set_threads(int n);

/* Philox4x32-10 of counter c[4] under key k[2] into out[4]. */
void or_philox4x32_10(const uint32_t c[4], const uint32_t k[2], uint32_t out[4]);

/* Fixed-point weight: weight * 2^shift rounded to nearest, ties to even. */
int64_t or_wfx(float w, int32_t shift);

/* The external Poisson counts the step loop draws for neurons 0..n-1 of a
 * population keyed `seed` over steps [step0, step0 + n_steps): out[steps][n]. */
void or_poisson_counts(const uint32_t *table, int32_t len, uint64_t seed, int64_t step0, int64_t n_steps,
                       int32_t n, int32_t *out);

/* Run steps [step0, step0 + n_steps) of the network in place: state, arrival
 * slots and rasters updated; *events += the synaptic events delivered.
 * Returns 0, or a negative code for an invalid description. */
int or_run(or_pop *pops, int32_t n_pops, const or_conn *conns, int32_t n_conns,
           int64_t step0, int64_t n_steps, uint64_t *events);

#ifdef __cplusplus
}
#endif
#endif
