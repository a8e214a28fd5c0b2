/*
 * naer2b -- the C ABI of the B200 hot path of naer2's per-timestep loop:
 * membrane update, spike-ring write and read, pull intake and push delivery,
 * stepped at a fixed dt and captured in CUDA graphs.
 *
 * Plain C: pointers, sizes and integers only. PyTorch (or any caller) owns
 * every device buffer; the library borrows the pointers for the lifetime of
 * a handle and allocates no device memory of its own (its tables live in the
 * caller's workspace, n2b_workspace_bytes; n2b_run_static uses a fixed array
 * inside the library instead). One handle = one network on one
 * device; calls on one handle are not thread-safe and must be serialised by
 * the caller; the work runs on the stream passed to each call.
 *
 * Error convention: every entry point returns 0 on success or a negative
 * N2B_E* code; n2b_last_error() returns the message of the calling thread's
 * last failure. Device-side faults of the data (an arrival slot or target
 * index out of range) are counted in the handle's error words
 * (n2b_status) instead of trapping.
 *
 * Each entry point names the reference interface it replaces
 * (MatteoSchmider/naer2, paths within that project).
 */
#ifndef NAER2B_H
#define NAER2B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define N2B_ABI_VERSION 2

/* return codes */
#define N2B_OK 0
#define N2B_EINVAL (-1)   /* an argument or description is invalid */
#define N2B_ECUDA (-2)    /* a CUDA call failed */
#define N2B_ESTATE (-3)   /* the call does not fit the handle's state */
#define N2B_ESPACE (-4)   /* the workspace is too small */

/* neuron models of the built-in kernels (a population's update and send) */
#define N2B_MODEL_LIF_DELTA 1      /* Brunel's time-driven LIF, delta synapses */
#define N2B_MODEL_PD14 2           /* PD14 LIF, exponential current synapses  */
#define N2B_MODEL_POISSON_SOURCE 3 /* independent Poisson spike source        */

/* how a connection's spikes reach its target */
#define N2B_PUSH 0 /* the source's block scatters its spikes into the target's arrival slots */
#define N2B_PULL 1 /* the target gathers its incoming links against the source's spike-bit ring */

/* error words (n2b_status) */
#define N2B_ERR_PUSH_LINK 0 /* push links with delay 0, delay >= arrival depth, or target >= n */
#define N2B_ERR_PULL_LINK 1 /* pull links with delay 0, delay >= bit depth, or source >= n */
#define N2B_ERR_SPLIT 2     /* push links past a row's split with a delay below 2 steps (skipped) */
#define N2B_ERR_ITEMS 3     /* work-list entries past its capacity (skipped; cannot happen for a valid split) */
#define N2B_ERR_BARRIER 4   /* persistent windows: a grid barrier wait that gave up (n2b_options.barrier_limit_ns,
                               default 2 s): the window stopped, and later windows return at once until
                               n2b_reset_counters */
#define N2B_ERR_PULL_STAGE 5 /* staged pull chunks that did not land within the wait limit (loaded directly
                                 instead; the launch stops staging) */
#define N2B_ERR_WORDS 8

/* One population: the state arrays and rings of the reference's
 * PopulationRuntime (naer2/runtime.py:213-290) at a fixed dt.
 * Model constants p[]:
 *   LIF_DELTA: p[0] decay = exp(-dt/tau_m) (fp32), p[1] theta, p[2] V_reset
 *   PD14:      p[0] P_V, p[1] P_I, p[2] P_VI, p[3] V_rest, p[4] V_thresh, p[5] V_reset
 *   POISSON_SOURCE: none (fire_threshold: fires when its uniform draw < it) */
typedef struct n2b_population {
    int32_t model;
    int32_t n;               /* neurons; at most 2^24 */
    int32_t acc_depth;       /* arrival slots: a power of two > every incoming delay (steps) */
    int32_t bit_depth;       /* spike-bit ring rows: a power of two > every outgoing pull delay, or 0 */
    int32_t shift;           /* fixed-point exponent of the summed input (0..62) */
    int32_t ref_steps;       /* refractory steps after a spike */
    uint32_t fire_threshold; /* POISSON_SOURCE only */
    int32_t ext_len;         /* entries of ext_table (0: no external Poisson drive) */
    uint64_t seed;           /* Philox key of the population's draws */
    int64_t ext_wfx;         /* fixed-point weight of one external Poisson event */
    float p[8];
    float *v;                /* [n] membrane potential (LIF_DELTA, PD14) */
    float *i;                /* [n] synaptic current (PD14) */
    int32_t *ref;            /* [n] refractory steps left (LIF_DELTA, PD14) */
    int64_t *acc;            /* [acc_depth][n] arrival slots, fixed point, zero at creation */
    uint32_t *bits;          /* [bit_depth][ceil(n/32)] spike-bit ring, or NULL */
    const uint32_t *ext_table; /* [ext_len] inverse-CDF table of the external Poisson count */
    uint32_t *raster;        /* [raster_steps][ceil(n/32)] recorded spike bits, or NULL */
    int64_t raster_steps;
} n2b_population;

/* One connection: the reference's SimulationTopology of one Connection
 * (naer2/topology.py:291-438, built by naer2/fabric.py:100-143), as CSR.
 * link[l] = (delay_steps << 24) | index, delay_steps in 1..255, index < 2^24:
 *   PUSH: rows per source neuron (ptr[n_src + 1]), index = target neuron;
 *   PULL: rows per target neuron (ptr[n_tgt + 1]), index = source neuron.
 * w: per-link weight, or NULL for `weight` on every link.
 * split (optional), PUSH: per source row, the first link of delay >= 2
 *   steps, the row's delay-1 links all before it. The spiking neuron's block
 *   delivers [ptr[s], split[s]) in the step itself; [split[s], ptr[s+1]) goes
 *   to a work list every block of the next step's launch shares. NULL: the
 *   spiking neuron's block delivers the whole row.
 * split (optional), PULL: [n_tgt + 1] row offsets of a second CSR in the same
 *   link array holding every link of delay >= 2 steps (split[0] >= ptr[n_tgt]):
 *   ptr's rows then hold only delay-1 links, pulled by the target's block in the
 *   step; split's rows are pulled one step ahead (at step n for the slot of step
 *   n + 1) by every warp of the launch in runs of 1024 links, each row's sum of a
 *   run added to its arrival slot with one reduction. NULL: ptr's rows hold every
 *   link, all pulled by the target's block in the step. */
typedef struct n2b_connection {
    int32_t src;
    int32_t tgt;
    int32_t mode;
    int32_t n_links;
    float weight;
    int32_t reserved;
    const int32_t *ptr;
    const uint32_t *link;
    const float *w;
    const int32_t *split;
} n2b_connection;

typedef struct n2b_options {
    int32_t block;   /* neurons (threads) per block: 64, 128 or 256 (0: 128) */
    int32_t device;  /* CUDA device ordinal of every pointer */
    int32_t grid;    /* blocks per launch (0: per-step launches two per SM and at least one per tile;
                        persistent one per SM, at least tiles + half an SM's worth, at most the co-resident
                        blocks, each looping over its tiles; persistent with a split pull connection or with
                        more tiles than two blocks per SM hold (the three-per-SM kernel): every co-resident
                        block) */
    int32_t persistent; /* 1: a window of steps is one cooperative launch, steps separated by a grid
                           barrier; 0: one launch per step */
    int32_t reserved;
    int64_t barrier_limit_ns; /* persistent windows: the longest a block waits at a grid barrier before the
                                 window stops with N2B_ERR_BARRIER (0: 2 s). Tests set a few ns: the wait
                                 then gives up at once although every block arrives, without a hang */
} n2b_options;

typedef struct n2b_net n2b_net;

/* The ABI version this library was built with (N2B_ABI_VERSION). */
int32_t n2b_abi_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char *n2b_last_error(void);

/* Device workspace bytes a network of this description needs (its tables,
 * step counter, error words and counters); 256-byte alignment required. */
int n2b_workspace_bytes(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns,
                        int32_t n_conns, const n2b_options *opt, size_t *bytes);

/* Build a network handle over the caller's buffers. Replaces
 * PopulationRuntime.__init__ + connect (naer2/runtime.py:216-311) and the
 * kernel build of FusedKernelTemplate.build (naer2/transpiler/templates/
 * fused_template.py:166-230): the kernels are compiled into this library.
 * The step counter starts at 0; the workspace is initialised on `stream`. */
int n2b_create(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
               const n2b_options *opt, void *workspace, size_t workspace_bytes, void *stream, n2b_net **out);

/* Advance n_steps steps of dt, one fused step kernel each. Replaces
 * PopulationRuntime.run / _launch (naer2/runtime.py:325-353, 506-526) as
 * Network.step drives them (naer2/network.py:80-152). */
int n2b_step(n2b_net *net, int64_t n_steps, void *stream);

/* Capture a window of `window_steps` steps into a CUDA graph (replacing any
 * earlier capture). Replaces WindowGraph's capture (naer2/graph.py:35-118). */
int n2b_capture(n2b_net *net, int32_t window_steps, void *stream);

/* Replay the captured window n_windows times (each advances window_steps
 * steps). Replaces WindowGraph.replay (naer2/graph.py:120-136). */
int n2b_replay(n2b_net *net, int64_t n_windows, void *stream);

/* Set the step counter (asynchronously, on `stream`); work of the previous
 * step still in the work list is dropped. */
int n2b_set_step(n2b_net *net, int64_t step, void *stream);

/* Start recording: raster row r of every population holds step step0 + r
 * (rows past raster_steps are not written). */
int n2b_record(n2b_net *net, int64_t step0, void *stream);

/* Copy the error words (N2B_ERR_*) into words[0 .. n_words) after the work
 * on `stream` (a synchronisation). Replaces PopulationRuntime.check and
 * Ring.check (naer2/runtime.py:724-735, naer2/ring.py:390-408). */
int n2b_status(n2b_net *net, int32_t *words, int32_t n_words, void *stream);

/* Copy the counters after the work on `stream` (a synchronisation):
 * out[0] synaptic events delivered, out[1] spikes, out[2 + p] spikes of
 * population p; n_out entries at most. Replaces the reference's
 * count_received counters (naer2/population.py:134-136). */
int n2b_counters(n2b_net *net, uint64_t *out, int32_t n_out, void *stream);

/* Zero the error words and counters, and clear a persistent window's abort
 * (on `stream`). */
int n2b_reset_counters(n2b_net *net, void *stream);

/* Release the handle (its graph; the caller's buffers stay the caller's). */
int n2b_destroy(n2b_net *net);

/* ---- Surrogate-gradient BPTT of a recurrent LIF layer --------------------
 * No counterpart in the reference (naer2 has no differentiable path): the
 * layer of the BPTT workload, hand-written forward and adjoint kernels.
 * Per sample and step t (dt = one step), hidden neuron i:
 *   Vpre = alpha V + U[t] + sum_in(i) w_k s[t - d_k][pre_k]   (d_k 1..5 steps)
 *   s    = Vpre >= theta (or, smooth, f(Vpre - theta), f(x) = x / (1 + slope |x|))
 *   V    = Vpre - theta s;   O[t] = beta O[t-1] + s W_out;   m = max over t of O
 * The backward uses g = 1 / (1 + slope |Vpre - theta|)^2 for ds/dVpre (the
 * fast-sigmoid surrogate; the exact derivative of the smooth f), the reset
 * included. The forward keeps the spikes of every step (one bit per neuron,
 * sample and step) and the membrane every `checkpoint` steps; the backward
 * recomputes each segment from its checkpoint, then runs it backwards over
 * the transposed (outgoing) rows. */

/* error words: 0 links with a bad code (skipped); 1 recomputed spikes that
 * differ from the forward's; 2 in_cta_max / out_cta_max below the rows' counts;
 * 3 waits of the backward's per-step exchange that gave up (the results are
 * then wrong; the kernel still ends) */
#define N2B_BPTT_ERR_WORDS 4

typedef struct n2b_bptt_desc {
    int32_t batch;       /* B, a multiple of 8 (8 samples per group of 8 CTAs) */
    int32_t steps;       /* T */
    int32_t hidden;      /* H, a multiple of 32, at most 1024 */
    int32_t readouts;    /* R, at most 32 */
    int32_t checkpoint;  /* K: membrane checkpoint every K steps */
    int32_t smooth;      /* 1: the smooth forward (hidden <= 256), for gradient checks */
    int32_t nnz;         /* recurrent links */
    int32_t in_cta_max;  /* most incoming links of any eighth of the hidden neurons */
    int32_t out_cta_max; /* most outgoing links of any eighth of the hidden neurons */
    float alpha, beta, theta, slope;
    const int32_t *in_ptr;    /* [H+1] incoming rows; the links' order is the weights' order */
    const uint16_t *in_code;  /* [nnz] source | delay << 11 */
    const int32_t *out_grp;   /* [H][6] outgoing rows: start of the delay-1..5 links, then the row end */
    const uint16_t *out_code; /* [nnz] target | delay << 11, outgoing order */
    const int32_t *out_perm;  /* [nnz] incoming-order index of each outgoing link */
    int32_t wait_polls;       /* polls before a backward exchange wait gives up with error word 3 (0: about a
                                 second); tests set a few, so that the wait gives up without a hang */
    int32_t reserved;
} n2b_bptt_desc;

/* Device workspace bytes of the layer (spike tape, checkpoints, one segment's
 * surrogate derivatives, per-group gradient partials). */
int n2b_bptt_workspace_bytes(const n2b_bptt_desc *d, size_t *bytes);

/* Forward over all steps: u [T][B][H] input current, w_rec [nnz] (incoming
 * order), w_out [H][R]; writes m [B][R] (max over time of the readouts) and
 * tstar [B][R] (its first step). tape = 1 keeps what the backward needs in
 * the workspace; 0 is the plain forward. */
int n2b_bptt_forward(const n2b_bptt_desc *d, const float *u, const float *w_rec, const float *w_out, int32_t tape,
                     float *m, int32_t *tstar, void *workspace, size_t workspace_bytes, void *stream);

/* Backward of the last taped forward: dm [B][R] = dL/dm, tstar as the forward
 * wrote it; writes du [T][B][H] = dL/du, dw_rec [nnz], dw_out [H][R]. The work
 * runs on two streams of the library's own (made on a device's first call,
 * kept): it starts after the work already on `stream`, and `stream` waits for
 * its end, so the results are ordered on `stream` as if it ran there. */
int n2b_bptt_backward(const n2b_bptt_desc *d, const float *u, const float *w_rec, const float *w_out,
                      const float *dm, const int32_t *tstar, float *du, float *dw_rec, float *dw_out,
                      void *workspace, size_t workspace_bytes, void *stream);

/* The N2B_BPTT_ERR_WORDS error words after the work on `stream` (a synchronisation). */
int n2b_bptt_status(const n2b_bptt_desc *d, void *workspace, size_t workspace_bytes, int32_t *words, void *stream);

/* Copy the taped spikes into out (device): [T][B/8][H] bytes, bit j = sample
 * 8c + j of group c; smooth: [T][B/8][H][8] floats. */
int n2b_bptt_spikes(const n2b_bptt_desc *d, void *workspace, size_t workspace_bytes, void *out, void *stream);

/* The layer's input projection over spike events (no counterpart in the
 * reference; it replaces a sparse-dense library product). Input row r is
 * sample b of step t (r = t * B + b); its spiking channels are
 * channel[row_ptr[r] .. row_ptr[r + 1]), ascending. Writes u [rows][hidden] =
 * the sum of those channels' rows of w_in [channels][hidden], in channel
 * order. hidden a multiple of 4 (at most 1024); w_in and u 16-byte aligned. */
int n2b_project_forward(const int32_t *row_ptr, const int32_t *channel, int32_t rows, int32_t channels,
                        int32_t hidden, const float *w_in, float *u, void *stream);

/* dw_in [channels][hidden] = x^T du for the same events, grouped by channel:
 * chunk k is the rows row_idx[chunk_ptr[k] .. chunk_ptr[k + 1]) (ascending,
 * one channel's), channel c owns chunks channel_chunk[c] .. channel_chunk[c + 1];
 * partials [n_chunks][hidden] is the caller's scratch. Each chunk is summed,
 * then each channel's chunks in order: the same result on every call. */
int n2b_project_backward(const int32_t *chunk_ptr, int32_t n_chunks, const int32_t *row_idx,
                         const int32_t *channel_chunk, int32_t channels, int32_t rows, int32_t hidden,
                         const float *du, float *partials, float *dw_in, void *stream);

/* ---- Run-time compiled step kernels of user-defined models ---------------
 * The transpiler (naer2_b200/transpiler) lowers a population's Python hooks
 * (receive / update / send) to CUDA device code inside a step-kernel template;
 * these entry points compile that source with NVRTC for the device's
 * architecture, load it and launch it. Replace the reference's
 * FusedKernelTemplate.build (naer2/transpiler/templates/fused_template.py:
 * 166-230, which builds a Triton/Gluon kernel) and its launch in
 * PopulationRuntime._launch (naer2/runtime.py:506-526). */
typedef struct n2b_jit_kernel n2b_jit_kernel;

/* Compile `source` (self-contained CUDA C++, no includes) and load its
 * extern "C" kernel `kernel_name` on `device`. options: extra NVRTC options.
 * A compile error returns N2B_EINVAL with NVRTC's log in n2b_last_error(). */
int n2b_jit_compile(const char *source, const char *kernel_name, const char *const *options, int32_t n_options,
                    int32_t device, n2b_jit_kernel **out);

/* Launch with one by-value parameter block of params_bytes bytes (the
 * kernel's single parameter), grid x block threads, on `stream`. */
int n2b_jit_launch(n2b_jit_kernel *k, uint32_t grid, uint32_t block, const void *params, size_t params_bytes,
                   void *stream);

/* A window of steps of a transpiled network in one call (the per-step loop of
 * naer2/network.py:80-152 over the populations' generated kernels): for each
 * step n = step0 .. step0 + n_steps - 1, and in it each kernel k in order, one
 * launch of kernels[k] (grids[k] x blocks[k] threads; grid 0: skipped) with a
 * copy of params[k] (params_bytes[k] >= 32) whose leading fields are set for
 * the step: the int64 step at offset 0 = n, the fp32 t at offset 24 =
 * (n + 1) dt and t0 at offset 28 = n dt, each rounded from double. */
int n2b_jit_launch_window(n2b_jit_kernel *const *kernels, const uint32_t *grids, const uint32_t *blocks,
                          const void *const *params, const size_t *params_bytes, int32_t n_kernels, int64_t step0,
                          int64_t n_steps, double dt, void *stream);

/* Unload the kernel. */
int n2b_jit_destroy(n2b_jit_kernel *k);

/* Size of the library's own device scratch used by n2b_run_static. */
#define N2B_STATIC_SCRATCH_BYTES ((size_t)32 << 20)

/* No counterpart in the reference: an addition of this library for callers
 * that cannot allocate device memory -- a host engine that reserves all of a
 * GPU's memory for its own pool up front (a cudaMalloc would fail or escape
 * its accounting), or code that must not call cudaMalloc / cudaFree because
 * they synchronise the whole device. It runs n_steps steps of the network
 * from step step0 (the step index the Poisson draws use), exactly as
 * n2b_create + n2b_set_step + n2b_record(step0) + n2b_step would on a
 * workspace, but with the workspace held in a file-scope device array of
 * N2B_STATIC_SCRATCH_BYTES bytes inside this library; it allocates no device
 * memory. The caller passes every input and output buffer, as for
 * n2b_create. The far links of the call's last step are delivered into the
 * arrival slots before the call's work ends, so a later call from step
 * step0 + n_steps continues the run exactly. If `status` is not NULL, the call
 * waits for its work on `stream` and copies the N2B_ERR_WORDS error words
 * there; with status NULL no error word is reported (a grid barrier that gave
 * up, or links out of range, pass unseen). Every call waits on `stream` for its
 * own set-up (it copies the network's tables into the array first), and it
 * makes `opt->device` current only for its own work: the caller's current
 * device is the same after the call.
 *
 * Limits: a network whose workspace (n2b_workspace_bytes) exceeds
 * N2B_STATIC_SCRATCH_BYTES is rejected with N2B_ESPACE. Every device that
 * loads this library holds the array until the process exits. Each call looks
 * the array's address up on the device it runs on. Every call on a device
 * shares the one array, and each call starts by resetting the counts, error
 * words and barrier in it: two calls whose work overlaps on the GPU (different
 * streams, or threads) race and corrupt each other. */
int n2b_run_static(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
                   const n2b_options *opt, int64_t step0, int64_t n_steps, int32_t *status, void *stream);

#ifdef __cplusplus
}
#endif
#endif
