// Device side of the fixed-dt hot path: Philox draws, the built-in neuron
// models, pull intake, and the fused step kernel. Written for sm_100a;
// included by naer2b.cu.
//
// One step n of a network, in one launch (step_kernel) or as one iteration of
// a persistent cooperative launch (persistent_kernel, steps separated by a
// bounded grid barrier). Tiles of NPB neurons of one population are spread
// over the blocks; every block then shares the far deliveries of step n - 1.
//   1. intake: each neuron's due arrival slot acc[n mod D][j] (int64 fixed
//      point, read and cleared), plus every pull connection's gather of its
//      incoming links (its delay-1 links where the connection is split)
//      against the source's spike-bit ring, plus the external Poisson events
//      -- all one exact integer sum, converted to float once;
//   2. the model's update and send (one thread per neuron);
//   3. spike-ring write: one __ballot_sync word per warp into the bit ring
//      (and the raster), the warp's spikes compacted with __popc into the
//      block's shared spike list;
//   4. near delivery: the block walks the delay-1 links of its own spikes
//      (the head of each outgoing row) as one flat (spike, link) range and
//      adds each weight into the target's slot (n + 1) mod D with a 64-bit
//      red.global.add; the rest of each row (delay >= 2) is cut into work
//      items of NPB links appended to this step's work list;
//   5. far delivery: every block takes items of step n - 1's list (grid
//      stride, from the last block down: blocks without a tile first), one
//      link per thread, into slots (n - 1 + delay) mod D, all >= n + 1:
//      never the slot this step reads;
//   6. the grid-wide pull: the delay >= 2 links of split pull connections,
//      gathered one step ahead for slot n + 1 (ring rows of steps <= n - 1),
//      in runs of PULL_ITEM links claimed by every warp of the grid, one
//      reduction per row a run finishes.
// Integer adds make every interleaving give the same sums. A step's slot is
// complete when it is read: the previous step ended (launch boundary or grid
// barrier) after every add into it.
//
// Latency is the budget here (a step moves ~1 MB): the tables of small
// networks ride in the kernel parameters (no dependent load before the state
// loads), each neuron's outgoing row bounds are loaded with its state, the
// Poisson inversion is a branch-free count over an inline table, and the far
// items are taken several at a time.
#pragma once
#include <stdint.h>

namespace n2b {

constexpr unsigned FULL = 0xffffffffu;
constexpr int INLINE_POPS = 32;   // populations whose tables fit the kernel parameters
constexpr int INLINE_PUSH = 64;
constexpr int INLINE_PULL = 16;
constexpr int EXT_INLINE = 32;    // Poisson table entries kept inline
constexpr int MERGE_OUT = 8;      // outgoing push connections walked together (more: one at a time)

// ------------------------------------------------------------------ tables

struct alignas(16) PopDev {
    int32_t model, n, acc_mask, bit_mask;      // masks: depth - 1
    int32_t words, shift, ref_steps, ext_len;
    uint32_t fire_threshold, seed_lo, seed_hi, index;
    int32_t out_first, n_out, pull_first, n_pull;
    long long ext_wfx;
    float inv_scale, pad0;
    float p[8];
    float *v;
    float *i;
    int32_t *ref;
    long long *acc;
    uint32_t *bits;
    const uint32_t *ext_table;
    uint32_t *raster;
    long long raster_steps;
    uint32_t ext_tab[EXT_INLINE];  // the table's first EXT_INLINE entries (all of it when ext_len <= EXT_INLINE)
};

struct alignas(16) ConnDev {
    int32_t homogeneous, src_n, tgt_n, tgt_acc_mask;
    int32_t src_bit_mask, src_words, has_split, staged;  // staged (pull): link (and w) 16-byte aligned
    long long wfx;        // homogeneous weight, fixed point of the target
    float wscale;         // 2^shift of the target (exact)
    int32_t item0;        // pull with split: its first item (PULL_ITEM links) of the grid-wide pull
    int32_t n_items;      // ... and its items (0: none)
    int32_t ring_off;     // pull: word offset of its source ring's copy in the ring cache (-1: not cached)
    int32_t far0;         // pull with split: the first delay >= 2 link (split[0])
    int32_t n_links;
    const int32_t *item_row;  // pull with split: each item's first row
    const int32_t *ptr;
    const uint32_t *link;
    const float *w;
    long long *tgt_acc;
    const uint32_t *src_bits;
    const int32_t *split;  // push: per source, its row's first link of delay >= 2 (NULL: none deferred);
                           // pull: the delay >= 2 rows' offsets (NULL: ptr's rows hold every link)
};

struct StepArgs {
    const PopDev *pops;    // global tables (always valid)
    const ConnDev *push;   // push connections, grouped by source population
    const ConnDev *pull;   // pull connections, grouped by target population
    const int4 *tiles;     // per tile: population, first neuron, neurons
    const long long *step; // the step counter (advanced after every launch)
    const long long *rec0; // raster row 0's step
    int32_t *err;
    unsigned long long *counters;
    int4 *items;           // 3 work lists of item_cap entries: (push connection, first link, end link, 0)
    int32_t *item_count;   // their lengths; step n appends to list n mod 3, reads n - 1's
    int32_t *tile_claim;   // per step n mod 3: tiles past the first gridDim.x claimed so far
    int32_t *pull_claim;   // per step n mod 3: grid-wide pull items past every warp's first claimed so far
    unsigned *barrier;     // persistent kernel: the arrival counter, the abort word
    unsigned long long *trace;  // N2B_TRACE builds: per step and block, %globaltimer at each phase (else unused)
    unsigned long long bar_limit_ns;  // persistent windows: a grid barrier wait gives up after this long
    int32_t trace_steps;
    int32_t pull_staged;   // the launch has a PullStage per warp in dynamic shared memory
    int32_t pull_stage_bytes;  // ... of this size each (pull_stage_bytes)
    int32_t ring_cache_words;  // ... and after them a copy of a pull source's spike-bit ring of at most this size
    int32_t ring_cache_all;    // every pull source's ring fits the cache at its ring_off (the grid-wide pull)
    int32_t pull_items;        // items of the grid-wide pull (the delay >= 2 rows, PULL_ITEM links each)
    int32_t n_pull;
    int32_t item_cap;
    int32_t n_tiles;
    int32_t offset;        // this launch's step = *step + offset (per-step launches)
    int32_t n_pops;
    int32_t n_push;
    int32_t tile_first[INLINE_POPS + 1];  // inline tables: population p owns tiles [tile_first[p], tile_first[p+1])
    PopDev pops_i[INLINE_POPS];
    ConnDev push_i[INLINE_PUSH];
    ConnDev pull_i[INLINE_PULL];
};

// Phase stamps of N2B_TRACE builds (the reference's TRACE levels, naer2/trace.py): step k's block b writes
// %globaltimer at phase p into trace[(k * gridDim.x + b) * TRACE_PHASES + p].
constexpr int TRACE_PHASES = 12;
#ifdef N2B_TRACE
#define N2B_STAMP(a, k, p)                                                                                   \
    do {                                                                                                     \
        if (threadIdx.x == 0 && (a).trace && (k) < (a).trace_steps) {                                        \
            unsigned long long _t;                                                                           \
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(_t));                                           \
            (a).trace[((size_t)(k) * gridDim.x + blockIdx.x) * TRACE_PHASES + (p)] = _t;                      \
        }                                                                                                    \
    } while (0)
#else
#define N2B_STAMP(a, k, p) \
    do {                   \
    } while (0)
#endif

template <bool INL>
__device__ __forceinline__ const PopDev &pop_at(const StepArgs &a, int k) {
    return INL ? a.pops_i[k] : a.pops[k];
}
template <bool INL>
__device__ __forceinline__ const ConnDev &push_at(const StepArgs &a, int k) {
    return INL ? a.push_i[k] : a.push[k];
}
template <bool INL>
__device__ __forceinline__ const ConnDev &pull_at(const StepArgs &a, int k) {
    return INL ? a.pull_i[k] : a.pull[k];
}

// (population, first neuron, neurons) of tile t
template <bool INL, int NPB>
__device__ __forceinline__ int4 tile_at(const StepArgs &a, int t) {
    if (!INL) return a.tiles[t];
    int p = 0;
    while (p + 1 < a.n_pops && a.tile_first[p + 1] <= t) ++p;
    const int first = (t - a.tile_first[p]) * NPB;
    return make_int4(p, first, min(NPB, a.pops_i[p].n - first), 0);
}

constexpr int BAR_COUNT = 0;      // persistent launches: arrivals of this launch's barriers
constexpr int BAR_ABORT = 32;     // set when a barrier wait gave up (a line of its own)
constexpr int BAR_WORDS = 64;
constexpr int BAR_MAX_BLOCKS = 1 << 16;
constexpr unsigned long long BAR_LIMIT_NS = 2000000000ull;  // default: a barrier wait gives up after 2 s

// ------------------------------------------------------------------ Philox

// Philox4x32-10 (Salmon et al., SC'11), first output word only: ten rounds of
// the two 32x32 -> 64 multiplies, the key bumped by the Weyl constants.
__device__ __forceinline__ uint32_t philox_word0(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                  uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c0;
}

// Neuron j's draw at step n, stream `purpose` (0: external drive, 1: source).
__device__ __forceinline__ uint32_t draw(const PopDev &P, int j, long long n, uint32_t purpose) {
    return philox_word0((uint32_t)j, (uint32_t)(unsigned long long)n,
                        (uint32_t)((unsigned long long)n >> 32), purpose, P.seed_lo, P.seed_hi);
}

// Poisson count by inversion: how many of the table's first len - 1 entries the uniform word reaches (the
// table is non-decreasing, so this is the first k with u < table[k]). Branch-free over the inline entries
// (uniform addresses across the warp), the rest from global memory.
__device__ __forceinline__ int poisson_count(const PopDev &P, uint32_t u) {
    const int last = P.ext_len - 1;
    int k = 0;
    const int m = min(last, EXT_INLINE);
#pragma unroll 8
    for (int q = 0; q < m; ++q) k += u >= P.ext_tab[q];
    for (int q = EXT_INLINE; q < last; ++q) k += u >= __ldg(P.ext_table + q);
    return k;
}

__device__ __forceinline__ long long weight_fx(float w, float wscale) {
    return __float2ll_rn(__fmul_rn(w, wscale));  // exact scale, nearest-even
}

// ------------------------------------------------------------------ warp / block helpers

__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ long long warp_incl_scan64(long long v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += u;
    }
    return v;
}

// Block-wide exclusive scan of one int64 per thread (NPB threads); the total in *total.
template <int NPB>
__device__ __forceinline__ long long block_excl_scan64(long long v, long long *s_wsum, long long *total) {
    constexpr int NW = NPB / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long incl = warp_incl_scan64(v);
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        long long x = lane < NW ? s_wsum[lane] : 0;
        x = warp_incl_scan64(x);
        if (lane < NW) s_wsum[lane] = x;
    }
    __syncthreads();
    *total = s_wsum[NW - 1];
    return incl - v + (warp > 0 ? s_wsum[warp - 1] : 0);
}

// Block-wide exclusive scan of one int per thread (NPB threads); the total in *total.
template <int NPB>
__device__ __forceinline__ int block_excl_scan(int v, int *s_wsum, int *total) {
    constexpr int NW = NPB / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int incl = warp_incl_scan(v);
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int x = lane < NW ? s_wsum[lane] : 0;
        x = warp_incl_scan(x);
        if (lane < NW) s_wsum[lane] = x;
    }
    __syncthreads();
    *total = s_wsum[NW - 1];
    return incl - v + (warp > 0 ? s_wsum[warp - 1] : 0);
}

// ------------------------------------------------------------------ models

// Brunel's time-driven LIF (tools/brunel_reference.py:36-42 of the reference):
// refractory neurons keep V and drop their input; otherwise V = V*decay + in,
// fire at V >= theta, reset, refractory for ref_steps.
__device__ __forceinline__ bool lif_delta(const PopDev &P, float in, float &v, int &ref) {
    if (ref > 0) {
        ref -= 1;
        return false;
    }
    v = __fadd_rn(__fmul_rn(v, P.p[0]), in);
    const bool fire = v >= P.p[1];
    if (fire) {
        v = P.p[2];
        ref = P.ref_steps;
    }
    return fire;
}

// PD14's LIF with exponential current synapses at fixed dt (reference
// test/networks/PD14/neuron.py:166-186): receive adds into the current, the
// exact propagators advance V and the current, threshold V > V_thresh.
__device__ __forceinline__ bool pd14(const PopDev &P, float in, float &v, float &cur, int &ref) {
    cur = __fadd_rn(cur, in);
    if (ref > 0) {
        ref -= 1;
        v = P.p[5];
    } else {
        const float a = __fmul_rn(P.p[0], __fsub_rn(v, P.p[3]));
        v = __fadd_rn(__fadd_rn(P.p[3], a), __fmul_rn(P.p[2], cur));
    }
    cur = __fmul_rn(P.p[1], cur);
    const bool fire = v > P.p[4];
    if (fire) {
        v = P.p[5];
        ref = P.ref_steps;
    }
    return fire;
}

// One synaptic event: a 64-bit reduction into an arrival slot, issued as a reduction (no value comes back).
// No memory clobber: nothing in the step reads an arrival slot after adding to it before the step's barrier
// (a grid barrier or the launch boundary), which orders the slot's reads.
__device__ __forceinline__ void red_add_u64(long long *p, long long v) {
    asm volatile("red.global.add.u64 [%0], %1;" ::"l"(p), "l"(v));
}

// ------------------------------------------------------------------ pull intake

// The pull (the reference's pull intake, fused.py:1626-1965): a warp sweeps one contiguous run of links of a
// pull CSR -- rows in target order -- in batches of 32 consecutive links, one per lane. Every lane follows its
// link's row by the row offsets (the row's end in a register) and looks its source's bit up in the spike-bit
// ring (copied to shared memory when small); the warp then sums the batch row by row without atomics: with a
// single weight the rows' spiking links are counted from a ballot (popc over each row's lanes), with per-link
// weights by a segmented shuffle scan. A row still open at the batch's end is carried in registers into the
// next batch, so every row of the run is handed on exactly once, by one lane, with its total.
// The run's links stream into shared memory by 1-D bulk copies (cp.async.bulk, completion counted on an
// mbarrier): PULL_CH links per chunk, PULL_BUFS chunks in flight. Only this GPU's own memory is read, and no
// copy is multicast. The run's 16-byte aligned interior is copied; its ragged head and tail (fewer than 4
// links each) are loaded directly, as is every link of a connection whose arrays are not 16-byte aligned.
// Two pulls use it: the delay-1 rows (every row without a split) by the target's own block in the step, for
// the warp's 32 neurons, and the delay >= 2 rows of split connections one step ahead, by every warp of the
// grid in runs of PULL_ITEM links (pull_far_phase).
constexpr int PULL_CH = 512;                        // links per staging chunk
constexpr int PULL_BUFS = 3;                        // chunks in flight per warp
constexpr int PULL_ITEM = 1024;                     // links per item of the grid-wide pull (a multiple of PULL_CH)
constexpr int RING_CACHE_MAX = 8192;                // words of pull sources' rings copied to shared memory, at most
constexpr unsigned PULL_WAIT_POLLS = 1u << 22;      // polls of a chunk's mbarrier before it counts as lost
constexpr int PULL_BATCH = 4;                       // batches whose link records are loaded together
static_assert(PULL_BATCH == 4, "a whole group inside the open row: four links per lane, one 16-byte load");
constexpr int PULL_SHORT_ROWS = 48;                 // in-step pull: rows this short on average, a lane per row

// One warp's staging area in dynamic shared memory: this header, then PULL_BUFS chunks of link records and,
// when the launch has a pull connection with per-link weights, PULL_BUFS chunks of weights.
struct alignas(16) PullStage {
    unsigned long long bar[PULL_BUFS];
    long long sum[32];          // the in-step pull: the warp's 32 rows' totals
    int32_t ptr[33];            // ... and their offsets
    uint32_t uses[PULL_BUFS];   // completions of each buffer's mbarrier so far (its next parity)
    int32_t broken;             // a chunk was lost: the rest of the launch loads links directly
};
constexpr size_t PULL_HEAD_BYTES = (sizeof(PullStage) + 15) & ~size_t(15);

__host__ __device__ constexpr size_t pull_stage_bytes(bool weighted) {
    return PULL_HEAD_BYTES + sizeof(uint32_t) * PULL_BUFS * PULL_CH * (weighted ? 2 : 1);
}

__device__ __forceinline__ uint32_t *stage_link(PullStage *st, int b) {
    return reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(st) + PULL_HEAD_BYTES) + b * PULL_CH;
}

__device__ __forceinline__ float *stage_w(PullStage *st, int b) {  // launches with weighted pull connections
    return reinterpret_cast<float *>(stage_link(st, PULL_BUFS)) + b * PULL_CH;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void pull_stage_init(PullStage *st) {
    if ((threadIdx.x & 31) == 0) {
        for (int b = 0; b < PULL_BUFS; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&st->bar[b])) : "memory");
            st->uses[b] = 0;
        }
        st->broken = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
}

// Lane 0: chunk k of the aligned range [a0, a1) into buffer k mod PULL_BUFS.
__device__ __forceinline__ void pull_issue(PullStage *st, const ConnDev &C, int a0, int a1, int k) {
    const int b = k % PULL_BUFS;
    const int c0 = a0 + k * PULL_CH, c1 = min(a1, c0 + PULL_CH);
    const uint32_t bytes = (uint32_t)(c1 - c0) * 4u;  // a multiple of 16: a0, a1 and PULL_CH are multiples of 4
    const uint32_t bar = smem_u32(&st->bar[b]);
    const uint32_t total = C.homogeneous ? bytes : 2u * bytes;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(total) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(stage_link(st, b))),
                 "l"(__cvta_generic_to_global(C.link + c0)), "r"(bytes), "r"(bar)
                 : "memory");
    if (!C.homogeneous)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32(stage_w(st, b))),
                     "l"(__cvta_generic_to_global(C.w + c0)), "r"(bytes), "r"(bar)
                     : "memory");
}

// Lane 0: the aligned range [a0, a1) (at most PULL_BUFS * PULL_CH links) into the stage's buffers taken as one,
// completion on buffer 0's mbarrier.
__device__ __forceinline__ void pull_issue_range(PullStage *st, const ConnDev &C, int a0, int a1) {
    const uint32_t bytes = (uint32_t)(a1 - a0) * 4u;  // a multiple of 16
    const uint32_t bar = smem_u32(&st->bar[0]);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(C.homogeneous ? bytes : 2u * bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(stage_link(st, 0))),
                 "l"(__cvta_generic_to_global(C.link + a0)), "r"(bytes), "r"(bar)
                 : "memory");
    if (!C.homogeneous)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_u32(stage_w(st, 0))),
                     "l"(__cvta_generic_to_global(C.w + a0)), "r"(bytes), "r"(bar)
                     : "memory");
}

// Every lane: wait (bounded) until buffer b's chunk has landed; false if it did not within the limit. Polls with
// the non-blocking mbarrier.test_wait.
__device__ __forceinline__ bool pull_wait(PullStage *st, int b) {
    const uint32_t bar = smem_u32(&st->bar[b]);
    const uint32_t parity = st->uses[b] & 1u;
    for (unsigned it = 0; it < 2 * PULL_WAIT_POLLS; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// One warp's sweep over a run of links of a pull CSR whose rows' offsets are `rows` (rows below qmax).
// HOMOG: one weight for every link; RING: the source's ring is the shared-memory copy.
// The open row (the row of the last link swept) is the same in every lane: a batch wholly inside it only adds
// each lane's spiking links (or their weights) to the lane's own part, with no exchange between lanes; a batch
// that reaches past it folds the parts into the row's total (one warp reduction) and sums the batch row by row.
template <bool HOMOG, bool RING>
struct PullPass {
    const uint32_t *ring;  // the source's spike-bit ring (shared-memory copy or global)
    const int32_t *rows;   // row offsets (global, or the warp's copy in shared memory)
    int nlo, mask, words, src_n, min_d, dspan, qmax;
    long long wfx;
    float wscale;
    int cq, cend;     // the open row and its end
    long long csum;   // its total, but for the lanes' parts since the last fold:
    long long lpart;  // per-link weights: the lane's part
    int lcnt;         // single weight: the lane's spiking links
    unsigned hits;    // links whose source spiked (the synaptic events of the pull)
    int bad;          // links out of range

    __device__ __forceinline__ uint32_t bits(uint32_t rec, bool valid, bool &ok) const {
        const int d = (int)(rec >> 24), s = (int)(rec & 0xFFFFFFu);
        // min_d <= d <= mask as one unsigned compare (dspan = mask - min_d; min_d 256 when no delay fits)
        ok = valid && (unsigned)(d - min_d) <= (unsigned)dspan && s < src_n;
        const int at = ((nlo - d) & mask) * words + (s >> 5);
        return ok ? (RING ? ring[at] : __ldcg(ring + at)) : 0u;
    }

    __device__ __forceinline__ void fold() {
        if (HOMOG) {
            hits += (unsigned)lcnt;  // (single weight: the parts are the hits)
            csum += (long long)__reduce_add_sync(FULL, (unsigned)lcnt) * wfx;
            lcnt = 0;
        } else {
            long long x = lpart;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(FULL, x, off);
            csum += x;
            lpart = 0;
        }
    }

    // A link of the open row into the lane's part.
    __device__ __forceinline__ void add(unsigned hit, float w) {
        if (HOMOG) {
            lcnt += (int)hit;
        } else {
            hits += hit;
            if (hit) lpart += weight_fx(w, wscale);
        }
    }

    // One link of a whole group inside the open row.
    __device__ __forceinline__ void open_link(uint32_t rec, float w) {
        bool ok;
        const uint32_t word = bits(rec, true, ok);  // 0 when the link is out of range
        bad += (int)!ok;
        add((word >> (rec & 31u)) & 1u, w);
    }

    // One batch (every lane of the warp): links [b, min(b + 32, r1)), the lane's link b + lane (`valid` below
    // r1) with its record, ring word and weight. emit(row, total) is called once per finished row, by one lane.
    template <class Emit>
    __device__ __forceinline__ void batch(int b, int r1, bool valid, uint32_t rec, uint32_t word, bool ok, float w,
                                          Emit &emit) {
        const int lane = threadIdx.x & 31;
        bad += (int)(valid && !ok);
        const unsigned hit = ok ? (word >> (rec & 31u)) & 1u : 0u;  // rec & 31 = s & 31
        if (min(b + 32, r1) <= cend) {  // the whole batch in the open row
            add(hit, w);
            return;
        }
        hits += hit;
        fold();
        int q = cq, end = cend;
        const int l = min(b + lane, r1 - 1);  // lanes past the batch's last link: that link
        while (l >= end && q + 1 < qmax) {    // rows may be empty
            ++q;
            end = rows[q + 1];
        }
        const int qn = __shfl_down_sync(FULL, q, 1);
        const unsigned ends = __ballot_sync(FULL, lane == 31 || qn != q);  // the last lane of every row
        if (cq != __shfl_sync(FULL, q, 0)) {  // the open row ended with the previous batch
            if (lane == 0) emit(cq, csum);
            csum = 0;
        }
        const unsigned below = ends & ((1u << lane) - 1u);
        const int start = below ? 32 - __clz(below) : 0;  // the first lane of the lane's row
        long long seg;
        if (HOMOG) {
            const unsigned m = ((2u << lane) - 1u) & ~((1u << start) - 1u);
            seg = (long long)__popc(__ballot_sync(FULL, hit != 0u) & m) * wfx;
        } else {
            seg = hit ? weight_fx(w, wscale) : 0;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {  // segmented inclusive scan
                const long long y = __shfl_up_sync(FULL, seg, off);
                if (lane - off >= start) seg += y;
            }
        }
        if (start == 0) seg += csum;  // the batch's first row continues the open row (csum is 0 otherwise)
        if (((ends >> lane) & 1u) && lane != 31) emit(q, seg);
        csum = __shfl_sync(FULL, seg, 31);
        cq = __shfl_sync(FULL, q, 31);
        cend = __shfl_sync(FULL, end, 31);
    }

    // The links [r0, r1) of the pass, their records at lk[l - base] (and weights at wk[l - base]): shared-memory
    // chunks (SMEM) or the connection's arrays (base 0), PULL_BATCH batches loaded together.
    template <bool SMEM, class Emit>
    __device__ __forceinline__ void run(const uint32_t *lk, const float *wk, int base, int r0, int r1, Emit &emit) {
        const int lane = threadIdx.x & 31;
        for (int b0 = r0; b0 < r1; b0 += 32 * PULL_BATCH) {
            if (SMEM) {
                // whole groups inside the open row: a lane takes four consecutive links per group (one 16-byte
                // load: lk is 16-byte aligned and b0 - base a multiple of 4), the order within a row being free
                const int lim = min(r1, cend);
                if (b0 + 32 * PULL_BATCH <= lim) {
                    for (; b0 + 32 * PULL_BATCH <= lim; b0 += 32 * PULL_BATCH) {
                        const uint4 r4 = *reinterpret_cast<const uint4 *>(lk + (b0 - base) + 4 * lane);
                        float4 w4 = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (!HOMOG) w4 = *reinterpret_cast<const float4 *>(wk + (b0 - base) + 4 * lane);
                        open_link(r4.x, w4.x);
                        open_link(r4.y, w4.y);
                        open_link(r4.z, w4.z);
                        open_link(r4.w, w4.w);
                    }
                    b0 -= 32 * PULL_BATCH;  // (the loop's increment)
                    continue;
                }
            }
            uint32_t rec[PULL_BATCH], word[PULL_BATCH];
            float w[PULL_BATCH];
            bool ok[PULL_BATCH];
#pragma unroll
            for (int k = 0; k < PULL_BATCH; ++k) {
                const int l = b0 + 32 * k + lane;
                rec[k] = 0u;
                w[k] = 0.f;
                if (l < r1) {
                    rec[k] = SMEM ? lk[l - base] : __ldg(lk + (l - base));
                    if (!HOMOG) w[k] = SMEM ? wk[l - base] : __ldg(wk + (l - base));
                }
            }
#pragma unroll
            for (int k = 0; k < PULL_BATCH; ++k) word[k] = bits(rec[k], b0 + 32 * k + lane < r1, ok[k]);
#pragma unroll
            for (int k = 0; k < PULL_BATCH; ++k)
                if (b0 + 32 * k < r1)
                    batch(b0 + 32 * k, r1, b0 + 32 * k + lane < r1, rec[k], word[k], ok[k], w[k], emit);
        }
    }
};

// The pass over links [L0, L1) (L0 < L1) of connection C, the first in row q0 of `rows` or a later one (rows
// before it empty), rows below qmax, against the ring rows of steps n_read - d (d >= min_d); each row the pass
// reaches goes to emit(row, total) once.
template <bool HOMOG, bool RING, class Emit>
__device__ __forceinline__ void pull_pass(const ConnDev &C, const uint32_t *ring, PullStage *st, int32_t *err,
                                          unsigned long long *events, const int32_t *rows, int q0, int qmax, int L0,
                                          int L1, long long n_read, int min_d, Emit &emit) {
    const int lane = threadIdx.x & 31;
    PullPass<HOMOG, RING> p;
    p.ring = ring;
    p.rows = rows;
    p.nlo = (int)n_read;  // the ring rows' index mod the depth: only the low bits matter
    p.mask = C.src_bit_mask;
    p.words = C.src_words;
    p.src_n = C.src_n;
    p.min_d = C.src_bit_mask >= min_d ? min_d : 256;  // (no 8-bit delay is 256 or more)
    p.dspan = C.src_bit_mask >= min_d ? C.src_bit_mask - min_d : 0;
    p.qmax = qmax;
    p.wfx = C.wfx;
    p.wscale = C.wscale;
    int q = q0, end = rows[q0 + 1];
    while (L0 >= end && q + 1 < qmax) {  // the row of link L0 (the same in every lane)
        ++q;
        end = rows[q + 1];
    }
    p.cq = q;
    p.cend = end;
    p.csum = 0;
    p.lpart = 0;
    p.lcnt = 0;
    p.hits = 0;
    p.bad = 0;
    const bool staged = C.staged && !__shfl_sync(FULL, st->broken, 0);  // lane 0 sets it: its value for all
    int a0 = (L0 + 3) & ~3, a1 = L1 & ~3;
    if (!staged || a1 <= a0) a0 = a1 = L1;  // nothing to stage: every link loaded directly
    const int n_chunks = (a1 - a0 + PULL_CH - 1) / PULL_CH;
    if (lane == 0)
        for (int k = 0; k < PULL_BUFS && k < n_chunks; ++k) pull_issue(st, C, a0, a1, k);
    p.template run<false>(C.link, C.w, 0, L0, a0, emit);  // the head (or every link)
    bool lost = false;
    for (int k = 0; k < n_chunks; ++k) {
        const int b = k % PULL_BUFS;
        const int c0 = a0 + k * PULL_CH, c1 = min(a1, c0 + PULL_CH);
        if (!lost) lost = __any_sync(FULL, !pull_wait(st, b));  // the same in every lane
        __syncwarp();
        if (lane == 0) st->uses[b] += 1;
        if (lost)  // a chunk that did not land in time: its links loaded directly
            p.template run<false>(C.link, C.w, 0, c0, c1, emit);
        else
            p.template run<true>(stage_link(st, b), HOMOG ? nullptr : stage_w(st, b), c0, c0, c1, emit);
        __syncwarp();  // every lane done with buffer b before it is refilled
        if (!lost && lane == 0 && k + PULL_BUFS < n_chunks) pull_issue(st, C, a0, a1, k + PULL_BUFS);
    }
    if (lost && lane == 0) {
        atomicAdd(err + 5, 1);
        st->broken = 1;
    }
    p.template run<false>(C.link, C.w, 0, max(a1, L0), L1, emit);  // the tail (fewer than 4 links)
    p.fold();
    if (lane == 0) emit(p.cq, p.csum);
    const unsigned hits = __reduce_add_sync(FULL, p.hits);
    const int bad = __reduce_add_sync(FULL, p.bad);
    if (lane == 0) {
        if (hits) atomicAdd(events, (unsigned long long)hits);
        if (bad) atomicAdd(err + 1, bad);
    }
}

template <bool RING, class Emit>
__device__ __forceinline__ void pull_pass_any(const ConnDev &C, const uint32_t *ring, PullStage *st, int32_t *err,
                                              unsigned long long *events, const int32_t *rows, int q0, int qmax,
                                              int L0, int L1, long long n_read, int min_d, Emit &emit) {
    if (C.homogeneous)
        pull_pass<true, RING>(C, ring, st, err, events, rows, q0, qmax, L0, L1, n_read, min_d, emit);
    else
        pull_pass<false, RING>(C, ring, st, err, events, rows, q0, qmax, L0, L1, n_read, min_d, emit);
}

// The launch's ring cache, after the warps' PullStages in dynamic shared memory.
__device__ __forceinline__ uint32_t *ring_cache(const StepArgs &a) {
    extern __shared__ __align__(128) unsigned char n2b_dyn_smem[];
    return reinterpret_cast<uint32_t *>(n2b_dyn_smem + (size_t)a.pull_stage_bytes * (blockDim.x >> 5));
}

// Words [first, first + count) of C's source ring into dst (at the same offsets), every thread of the block;
// 16-byte loads where both sides allow them, several in flight per thread.
__device__ __forceinline__ void copy_ring(uint32_t *dst, const ConnDev &C, int first, int count) {
    const uint32_t *s = C.src_bits + first;
    uint32_t *d = dst + first;
    if ((((uintptr_t)s | (uintptr_t)d) & 15u) == 0 && (count & 3) == 0) {
        const uint4 *s4 = reinterpret_cast<const uint4 *>(s);
        uint4 *d4 = reinterpret_cast<uint4 *>(d);
#pragma unroll 4
        for (int k = threadIdx.x; k < (count >> 2); k += blockDim.x) d4[k] = __ldcg(s4 + k);
    } else {
#pragma unroll 4
        for (int k = threadIdx.x; k < count; k += blockDim.x) d[k] = __ldcg(s + k);
    }
}

// The in-step pull over short rows: lane q sums row q alone (links [r0, r1) of C, in order, four loads in
// flight), no exchange between lanes; lanes without a row pass r0 = r1. Links [a0, a1) are read from the
// stage's buffers (st non-null: the warp's staged range), the others from C's arrays. Returns the row total.
template <bool HOMOG, bool RING>
__device__ __forceinline__ long long pull_lane_row(const ConnDev &C, const uint32_t *ring, int32_t *err,
                                                   unsigned long long *events, int r0, int r1, long long n_read,
                                                   PullStage *st, int a0, int a1) {
    const uint32_t *slink = st ? stage_link(st, 0) : nullptr;
    const float *sw = (st && !HOMOG) ? stage_w(st, 0) : nullptr;
    PullPass<HOMOG, RING> p;  // (its ring lookup only)
    p.ring = ring;
    p.nlo = (int)n_read;
    p.mask = C.src_bit_mask;
    p.words = C.src_words;
    p.src_n = C.src_n;
    p.min_d = C.src_bit_mask >= 1 ? 1 : 256;
    p.dspan = C.src_bit_mask >= 1 ? C.src_bit_mask - 1 : 0;
    long long part = 0;
    int cnt = 0, bad = 0;
    unsigned hits = 0;
    for (int l = r0; l < r1; l += 4) {
        uint32_t rec[4], word[4];
        float w[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = l + k;
            const bool in_stage = slink != nullptr && m >= a0 && m < a1;
            rec[k] = m < r1 ? (in_stage ? slink[m - a0] : __ldg(C.link + m)) : 0u;
            w[k] = (!HOMOG && m < r1) ? (in_stage ? sw[m - a0] : __ldg(C.w + m)) : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) word[k] = p.bits(rec[k], l + k < r1, ok[k]);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            bad += (int)(l + k < r1 && !ok[k]);
            const unsigned hit = ok[k] ? (word[k] >> (rec[k] & 31u)) & 1u : 0u;
            hits += hit;
            if (HOMOG) cnt += (int)hit;
            else if (hit) part += weight_fx(w[k], C.wscale);
        }
    }
    hits = __reduce_add_sync(FULL, hits);
    bad = __reduce_add_sync(FULL, bad);
    if ((threadIdx.x & 31) == 0) {
        if (hits) atomicAdd(events, (unsigned long long)hits);
        if (bad) atomicAdd(err + 1, bad);
    }
    return HOMOG ? (long long)cnt * C.wfx : part;
}

template <bool RING>
__device__ __forceinline__ long long pull_lane_row_any(const ConnDev &C, const uint32_t *ring, int32_t *err,
                                                       unsigned long long *events, int r0, int r1, long long n_read,
                                                       PullStage *st, int a0, int a1) {
    return C.homogeneous ? pull_lane_row<true, RING>(C, ring, err, events, r0, r1, n_read, st, a0, a1)
                         : pull_lane_row<false, RING>(C, ring, err, events, r0, r1, n_read, st, a0, a1);
}

// The in-step pull of the tile's population (every thread of the block): each pull connection's rows of ptr --
// all its links, or, with a split, its delay-1 links -- for the warp's 32 neurons, against ring rows n - d;
// returns the lane's own neuron's total. A source whose whole ring fits the ring cache is copied there first:
// with a split only ring row n - 1 (the delay-1 links' row), else the whole ring (its rows of steps before n are
// final). The warp's row offsets are copied to its PullStage; rows shorter than PULL_SHORT_ROWS links on
// average are summed a lane per row (their links staged by one bulk copy, issued before the ring's copy), longer
// ones swept by the whole warp (pull_pass).
template <bool INL>
__device__ __forceinline__ long long pull_intake(const StepArgs &a, const PopDev &P, int first, int count,
                                                 long long n, PullStage *stage) {
    const int lane = threadIdx.x & 31;
    const int wbase = first + (threadIdx.x & ~31);
    const int nq = min(32, first + count - wbase);
    long long mine = 0;
    for (int c = P.pull_first; c < P.pull_first + P.n_pull; ++c) {
        const ConnDev &C = pull_at<INL>(a, c);
        const int ring_words = (C.src_bit_mask + 1) * C.src_words;
        const bool cached = ring_words <= a.ring_cache_words;  // the same for every thread of the block
        uint32_t *cache = ring_cache(a);
        // (a network with pull connections always has its PullStages: the launch's dynamic shared memory)
        int L0 = 0, L1 = 0, a0 = 0, a1 = 0;
        bool short_rows = false, pre = false;
        if (nq > 0) {
            if (lane <= nq) stage->ptr[lane] = __ldg(C.ptr + wbase + lane);
            if (lane == 0 && nq == 32) stage->ptr[32] = __ldg(C.ptr + wbase + 32);
            stage->sum[lane] = 0;
            __syncwarp();
            L0 = stage->ptr[0];
            L1 = stage->ptr[nq];
            short_rows = L1 - L0 < PULL_SHORT_ROWS * nq;  // the same for every lane
            // short rows: the warp's whole range (its aligned interior) in one copy, in flight under the ring's
            a0 = (L0 + 3) & ~3;
            a1 = L1 & ~3;
            pre = short_rows && C.staged && a1 > a0 && a1 - a0 <= PULL_BUFS * PULL_CH &&
                  !__shfl_sync(FULL, stage->broken, 0);
            if (pre && lane == 0) pull_issue_range(stage, C, a0, a1);
        }
        if (cached) {
            __syncthreads();  // every warp done with the cache's previous ring
            if (C.has_split)
                copy_ring(cache, C, (int)((n - 1) & C.src_bit_mask) * C.src_words, C.src_words);
            else
                copy_ring(cache, C, 0, ring_words);
            __syncthreads();
        }
        if (nq <= 0) continue;
        if (short_rows) {  // a lane per row
            bool lost = false;
            if (pre) {
                lost = __any_sync(FULL, !pull_wait(stage, 0));  // the same in every lane
                __syncwarp();
                if (lane == 0) {
                    stage->uses[0] += 1;
                    if (lost) {
                        atomicAdd(a.err + 5, 1);
                        stage->broken = 1;
                    }
                }
            }
            PullStage *from = (pre && !lost) ? stage : nullptr;
            const int r0 = lane < nq ? stage->ptr[lane] : 0, r1 = lane < nq ? stage->ptr[lane + 1] : 0;
            mine += cached ? pull_lane_row_any<true>(C, cache, a.err, a.counters, r0, r1, n, from, a0, a1)
                           : pull_lane_row_any<false>(C, C.src_bits, a.err, a.counters, r0, r1, n, from, a0, a1);
        } else if (L1 > L0) {  // the warp sweeps the rows together
            auto emit = [&](int q, long long v) { stage->sum[q] = v; };  // q: the warp's row, below nq
            if (cached)
                pull_pass_any<true>(C, cache, stage, a.err, a.counters, stage->ptr, 0, nq, L0, L1, n, 1, emit);
            else
                pull_pass_any<false>(C, C.src_bits, stage, a.err, a.counters, stage->ptr, 0, nq, L0, L1, n, 1,
                                     emit);
            __syncwarp();
            mine += stage->sum[lane];
        }
        __syncwarp();  // every lane done with the stage before its next use
    }
    return lane < nq ? mine : 0;
}

// The grid-wide pull (every thread of every block, after the step's far items): the delay >= 2 rows of every
// split pull connection, for the arrival slot of step n + 1 -- ring rows (n + 1) - d, d >= 2, all written
// before this step -- in items of PULL_ITEM links (item k of a connection: its links [PULL_ITEM (k0 + k),
// PULL_ITEM (k0 + k + 1)) within the delay >= 2 region, k0 = far0 / PULL_ITEM; its first row in item_row[k]),
// every warp taking item (its index in the grid) first, then the step's next unclaimed one until none is left
// (blocks whose tiles took longer take fewer). Each row an item finishes is added to its slot with one reduction (slot n + 1
// is read after the step's barrier). With every pull source's ring in the cache together, the block copies them
// all first.
template <int NPB, bool INL>
__device__ __forceinline__ void pull_far_phase(const StepArgs &a, const long long n, PullStage *stage) {
    if (a.pull_items == 0 || stage == nullptr) return;  // the same for every thread of the launch
    uint32_t *cache = ring_cache(a);
    if (a.ring_cache_all) {
        __syncthreads();
        for (int c = 0; c < a.n_pull; ++c) {
            const ConnDev &C = pull_at<INL>(a, c);
            bool first = C.n_items > 0 && C.ring_off >= 0;  // connections of one source share its copy
            for (int e = 0; first && e < c; ++e)
                first = !(pull_at<INL>(a, e).n_items > 0 && pull_at<INL>(a, e).ring_off == C.ring_off);
            if (first) copy_ring(cache + C.ring_off, C, 0, (C.src_bit_mask + 1) * C.src_words);
        }
        __syncthreads();
    }
    const int W = (int)gridDim.x * (NPB / 32);
    int *claim = a.pull_claim + (int)(n % 3);
    int c = 0;
    for (int it = (int)blockIdx.x * (NPB / 32) + (int)(threadIdx.x >> 5); it < a.pull_items;) {
        int next = 0;
        if ((threadIdx.x & 31) == 0) next = W + atomicAdd(claim, 1);  // the warp's next item, in flight under this one
        while (c + 1 < a.n_pull && !(it >= pull_at<INL>(a, c).item0 &&
                                     it < pull_at<INL>(a, c).item0 + pull_at<INL>(a, c).n_items))
            ++c;  // a warp's items rise, and with them the connection index: the search moves forward only
        const ConnDev &C = pull_at<INL>(a, c);
        const int k = it - C.item0, k0 = C.far0 / PULL_ITEM;
        const int L0 = max(C.far0, (k0 + k) * PULL_ITEM), L1 = min(C.n_links, (k0 + k + 1) * PULL_ITEM);
        it = __shfl_sync(FULL, next, 0);
        if (L1 <= L0) continue;
        long long *slot = C.tgt_acc + (size_t)((n + 1) & C.tgt_acc_mask) * (size_t)C.tgt_n;
        auto emit = [&](int q, long long v) {
            if (v) red_add_u64(slot + q, v);
        };
        const int q0 = __ldg(C.item_row + k);
        if (a.ring_cache_all && C.ring_off >= 0)
            pull_pass_any<true>(C, cache + C.ring_off, stage, a.err, a.counters, C.split, q0, C.tgt_n, L0, L1, n + 1,
                                2, emit);
        else
            pull_pass_any<false>(C, C.src_bits, stage, a.err, a.counters, C.split, q0, C.tgt_n, L0, L1, n + 1, 2,
                                 emit);
    }
}

// Set-up: the first row of every item of a split pull connection's grid-wide pull -- the row r holding link
// PULL_ITEM (k0 + k) (or far0, for item 0), the last r with split[r] <= that link.
__global__ void pull_item_rows_kernel(const int32_t *split, int32_t tgt_n, int32_t far0, int32_t n_items,
                                      int32_t *item_row) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_items) return;
    const int l = max(far0, (far0 / PULL_ITEM + k) * PULL_ITEM);
    int lo = 0, hi = tgt_n;  // split[lo] <= l (split[0] = far0); answer in [lo, hi)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (split[mid] <= l) lo = mid;
        else hi = mid;
    }
    item_row[k] = lo;
}

// ------------------------------------------------------------------ delivery

// What delivering a push link needs of its connection, compact: the launch copies it into shared memory
// (every lane of a walk may look up a different connection; shared memory serves that in one pass, the
// parameter space's constant cache would serialize it).
struct SConn {
    long long *tgt_acc;
    const uint32_t *link;
    const float *w;
    long long wfx;
    float wscale;
    int32_t tgt_n, tgt_acc_mask, homogeneous;
};
constexpr int SMEM_CONNS = 64;  // push connections whose SConn the launch keeps in shared memory

__device__ __forceinline__ SConn sconn_of(const ConnDev &C) {
    SConn s;
    s.tgt_acc = C.tgt_acc;
    s.link = C.link;
    s.w = C.w;
    s.wfx = C.wfx;
    s.wscale = C.wscale;
    s.tgt_n = C.tgt_n;
    s.tgt_acc_mask = C.tgt_acc_mask;
    s.homogeneous = C.homogeneous;
    return s;
}

// Push connection c's SConn: from the launch's shared table, or (more connections than it holds) global memory.
__device__ __forceinline__ SConn conn_view(const StepArgs &a, const SConn *s_conn, int c) {
    return s_conn ? s_conn[c] : sconn_of(a.push[c]);
}

// Fill the shared table (every thread of the block, before a barrier).
template <bool INL>
__device__ __forceinline__ const SConn *fill_conns(const StepArgs &a, SConn *s_conn, int n_push) {
    if (n_push > SMEM_CONNS) return nullptr;
    for (int c = threadIdx.x; c < n_push; c += blockDim.x) s_conn[c] = sconn_of(push_at<INL>(a, c));
    return s_conn;
}

// Link l's per-link weight (0 for a single-weight connection), loaded with its link word, not after it.
template <class C_>
__device__ __forceinline__ float link_weight(const C_ &C, int l) {
    return C.homogeneous ? 0.f : __ldg(C.w + l);
}


// One link word (and its weight) into the target's arrival slot (n + delay) mod D; out-of-range links
// counted, not written.

template <class C_>
__device__ __forceinline__ void deliver_rec(const StepArgs &a, const C_ &C, uint32_t rec, float w, long long n,
                                            int min_delay) {
    const int d = (int)(rec >> 24), t = (int)(rec & 0xFFFFFFu);
    if (d < min_delay) {
        atomicAdd(a.err + 2, 1);  // a deferred link below 2 steps would land in a slot already read
        return;
    }
    if (d > C.tgt_acc_mask || t >= C.tgt_n) {
        atomicAdd(a.err + 0, 1);
        return;
    }
    const long long wfx = C.homogeneous ? C.wfx : weight_fx(w, C.wscale);
    red_add_u64(C.tgt_acc + (size_t)((n + d) & C.tgt_acc_mask) * (size_t)C.tgt_n + t, wfx);
}

// Row bounds of neuron j in an outgoing push connection: first link, split, end.
struct Row {
    int r0, sp, r1;
};

__device__ __forceinline__ Row row_of(const ConnDev &C, int j) {
    Row r;
    r.r0 = __ldg(C.ptr + j);
    r.r1 = __ldg(C.ptr + j + 1);
    r.sp = C.has_split ? min(max(__ldg(C.split + j), r.r0), r.r1) : r.r1;
    return r;
}

// A block's shared scratch of one tile phase (declared once per kernel).
template <int NPB>
struct Scratch {
    int cnt;
    int spk[NPB];                      // the tile's spiking neurons (population indices), compacted
    int row[NPB + 1];                  // connections past MERGE_OUT: per spike its row start
    int off[NPB + 1];                  // ... and its near-link offsets
    int wsum[NPB / 32];
    int w_pref[NPB / 32][MERGE_OUT + 1];  // per warp: its spike's near links, prefix over connections
    int w_r0[NPB / 32][MERGE_OUT];        // per warp: its spike's row start per connection
};

// The block's spikes, one warp per spike, its first MERGE_OUT outgoing push connections at once. Lane c holds
// connection c's row bounds (from shared memory for a persistent block's own tile, else one round trip);
// lane 0 claims the spike's far items with one atomic, issued before the walk and used after it; the warp
// walks the spike's delay-1 links of every connection as one flat range, NEAR_BATCH loads per lane issued
// before their reductions (an in-order issue would otherwise wait on each load before the next).
constexpr int NEAR_BATCH = 4;

template <int NPB, bool INL>
__device__ __forceinline__ void deliver_spikes(const StepArgs &a, const PopDev &P, int tile_y, const int *s_cache,
                                               int cnt, long long n, Scratch<NPB> &sc, const SConn *s_conn,
                                               int k = 0) {
    constexpr int NW = NPB / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m = min(P.n_out, MERGE_OUT);
    int *pref = sc.w_pref[warp], *r0s = sc.w_r0[warp];
    // fewer spikes than warps: each spike's walk split over a group of g warps (g a power of two)
    int g = 1;
    while (2 * g * cnt <= NW) g *= 2;
    const int sub = warp % g;
    for (int p = warp / g; p < cnt; p += NW / g) {
        const int jj = sc.spk[p];
        Row r = Row{0, 0, 0};
        if (lane < m) {
            if (s_cache) {
                const int t = jj - tile_y;
                r = Row{s_cache[(3 * lane) * NPB + t], s_cache[(3 * lane + 1) * NPB + t], s_cache[(3 * lane + 2) * NPB + t]};
            } else {
                r = row_of(push_at<INL>(a, P.out_first + lane), jj);
            }
        }
        const int near_c = r.sp - r.r0;
        const int items_c = (r.r1 - r.sp + NPB - 1) / NPB;
        const int items_incl = warp_incl_scan(items_c);
        const int near_incl = warp_incl_scan(near_c);
        const int total_items = __shfl_sync(FULL, items_incl, 31);
        const int total_near = __shfl_sync(FULL, near_incl, 31);
        const int links = __reduce_add_sync(FULL, r.r1 - r.r0);
        int base = 0;
        if (lane == 0 && sub == 0) {  // the group's first warp claims the items and counts the events
            if (total_items > 0) base = atomicAdd(a.item_count + (int)(n % 3), total_items);
            if (links) atomicAdd(a.counters + 0, (unsigned long long)links);
        }
        if (lane < m) {
            pref[lane] = near_incl - near_c;
            r0s[lane] = r.r0;
        }
        if (lane == 0) pref[m] = total_near;
        __syncwarp();
        for (int b0 = sub * 32; b0 < total_near; b0 += 32 * g * NEAR_BATCH) {
            uint32_t rec[NEAR_BATCH];
            float w[NEAR_BATCH];
            int cc[NEAR_BATCH];
#pragma unroll
            for (int b = 0; b < NEAR_BATCH; ++b) {
                const int idx = b0 + b * 32 * g + lane;
                cc[b] = -1;
                if (idx < total_near) {
                    int c = 0;
                    while (c + 1 < m && pref[c + 1] <= idx) ++c;
                    const SConn C = conn_view(a, s_conn, P.out_first + c);
                    const int l = r0s[c] + (idx - pref[c]);
                    rec[b] = __ldg(C.link + l);
                    w[b] = link_weight(C, l);
                    cc[b] = c;
                }
            }
#pragma unroll
            for (int b = 0; b < NEAR_BATCH; ++b)
                if (cc[b] >= 0) deliver_rec(a, conn_view(a, s_conn, P.out_first + cc[b]), rec[b], w[b], n, 1);
        }
        __syncwarp();
        if (sub == 0) {
            base = __shfl_sync(FULL, base, 0);
            if (lane < m && items_c > 0) {
                int at = base + items_incl - items_c;
                int4 *list = a.items + (size_t)(n % 3) * (size_t)a.item_cap;
                for (int q = r.sp; q < r.r1; q += NPB, ++at) {
                    if (at < a.item_cap) list[at] = make_int4(P.out_first + lane, q, min(q + NPB, r.r1), 0);
                    else atomicAdd(a.err + 3, 1);
                }
            }
        }
    }
}

// Connections past the first MERGE_OUT: one at a time, their rows loaded on demand.
template <int NPB, bool INL>
__device__ __forceinline__ void deliver_spikes_one(const StepArgs &a, const ConnDev &C, int c, const Row &row,
                                                   bool fire, int pos, int cnt, long long n, int *s_row, int *s_off,
                                                   int *s_wsum) {
    const int tid = threadIdx.x, lane = tid & 31;
    const int row_len = fire ? row.r1 - row.r0 : 0;
    const int warp_links = __reduce_add_sync(FULL, row_len);
    if (lane == 0 && warp_links) atomicAdd(a.counters + 0, (unsigned long long)warp_links);
    int n_items = 0, at = 0;
    if (fire) {
        s_row[pos] = row.r0;
        s_off[pos] = row.sp - row.r0;
        n_items = (row.r1 - row.sp + NPB - 1) / NPB;
        if (n_items > 0) at = atomicAdd(a.item_count + (int)(n % 3), n_items);
    }
    __syncthreads();
    const int near = tid < cnt ? s_off[tid] : 0;
    int total = 0;
    const int off = block_excl_scan<NPB>(near, s_wsum, &total);
    if (tid < cnt) s_off[tid] = off;
    if (tid == 0) s_off[cnt] = total;
    __syncthreads();
    for (int idx = tid; idx < total; idx += NPB) {
        int lo = 0, hi = cnt;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_off[mid] <= idx) lo = mid; else hi = mid;
        }
        const int l = s_row[lo] + (idx - s_off[lo]);
        deliver_rec(a, C, __ldg(C.link + l), link_weight(C, l), n, 1);
    }
    if (n_items > 0) {
        int4 *list = a.items + (size_t)(n % 3) * (size_t)a.item_cap;
        for (int k = 0; k < n_items; ++k) {
            if (at + k < a.item_cap) {
                const int l0 = row.sp + k * NPB;
                list[at + k] = make_int4(c, l0, min(l0 + NPB, row.r1), 0);
            } else {
                atomicAdd(a.err + 3, 1);
            }
        }
    }
    __syncthreads();
}

// ------------------------------------------------------------------ one tile of one step

// A neuron's state as its thread holds it through a step: membrane, current, refractory count. A
// persistent launch keeps its block's first tile here (and that tile's row bounds in shared memory) for the
// whole window.
struct Neuron {
    float v, cur;
    int ref;
};

__device__ __forceinline__ void load_neuron(const PopDev &P, int j, bool live, Neuron &nr) {
    nr.v = 0.f;
    nr.cur = 0.f;
    nr.ref = 0;
    if (!live || P.model == 3) return;
    nr.v = P.v[j];
    nr.ref = P.ref[j];
    if (P.model == 2) nr.cur = P.i[j];
}

__device__ __forceinline__ void store_neuron(const PopDev &P, int j, bool live, const Neuron &nr) {
    if (!live || P.model == 3) return;
    P.v[j] = nr.v;
    P.ref[j] = nr.ref;
    if (P.model == 2) P.i[j] = nr.cur;
}

// The row bounds of a tile's neurons in its first MERGE_OUT outgoing connections, into shared memory:
// s_cache[(3c + 0/1/2) * NPB + thread] = first link / split / end of connection c's row.
template <int NPB, bool INL>
__device__ __forceinline__ void cache_rows(const StepArgs &a, const PopDev &P, int j, bool live, int *s_cache) {
    const int m = min(P.n_out, MERGE_OUT);
    for (int c = 0; c < m; ++c) {
        const Row r = live ? row_of(push_at<INL>(a, P.out_first + c), j) : Row{0, 0, 0};
        s_cache[(3 * c) * NPB + threadIdx.x] = r.r0;
        s_cache[(3 * c + 1) * NPB + threadIdx.x] = r.sp;
        s_cache[(3 * c + 2) * NPB + threadIdx.x] = r.r1;
    }
}

// One tile of one step. CACHED: the tile's Neuron is held in registers by the caller across steps (loaded
// before the window, stored after it) and its row bounds are in s_cache; otherwise both come from memory.
template <int NPB, bool INL, bool CACHED, bool PULL>
__device__ __forceinline__ void tile_phase(const StepArgs &a, const long long n, const int4 tile, int k, Neuron &nr,
                                           const int *s_cache, Scratch<NPB> &sc, const SConn *s_conn,
                                           PullStage *stage) {
    int &s_cnt = sc.cnt;
    int *s_row = sc.row, *s_off = sc.off, *s_wsum = sc.wsum;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const PopDev &P = pop_at<INL>(a, tile.x);
    const int j = tile.y + tid;
    const bool live = tid < tile.z;
    __syncthreads();  // a block's previous tile: every thread past its reads of the shared arrays
    if (tid == 0) s_cnt = 0;

    // the arrival slot (and, uncached, the state: the loads do not wait for each other)
    const int model = P.model;
    long long acc = 0;
    long long *slot = nullptr;
    if (live && model != 3) {
        slot = P.acc + (size_t)(n & P.acc_mask) * (size_t)P.n + j;
        acc = __ldcg(slot);  // L2: other blocks' adds of this kernel are there, not in this SM's L1
    }
    if (!CACHED) load_neuron(P, j, live, nr);
    float &v = nr.v, &cur = nr.cur;
    int &ref = nr.ref;
    const int n_out = P.n_out;

    // 1-2. intake and update
    bool fire = false;
    if (model == 3) {  // N2B_MODEL_POISSON_SOURCE
        fire = live && draw(P, j, n, 1u) < P.fire_threshold;
    } else {
        if (PULL && P.n_pull > 0) acc += pull_intake<INL>(a, P, tile.y, tile.z, n, stage);
        if (live) {
            *slot = 0;
            if (P.ext_len > 0) acc += (long long)poisson_count(P, draw(P, j, n, 0u)) * P.ext_wfx;
            const float in = __fmul_rn(__ll2float_rn(acc), P.inv_scale);
            fire = (model == 1) ? lif_delta(P, in, v, ref) : pd14(P, in, v, cur, ref);
        }
        if (!CACHED) store_neuron(P, j, live, nr);
    }

    // 3. spike ring: a ballot word per warp, the spikes compacted into shared memory
    const uint32_t b = __ballot_sync(FULL, fire);
    if (lane == 0 && tile.y + warp * 32 < P.n) {
        const int w = (tile.y >> 5) + warp;
        if (P.bits) P.bits[(size_t)(n & P.bit_mask) * P.words + w] = b;
        if (P.raster) {
            const long long row = n - *a.rec0;
            if (row >= 0 && row < P.raster_steps) P.raster[(size_t)row * P.words + w] = b;
        }
    }
    __syncthreads();
    int base = 0;
    if (lane == 0 && b) base = atomicAdd(&s_cnt, __popc(b));
    base = __shfl_sync(FULL, base, 0);
    const int pos = base + __popc(b & ((1u << lane) - 1u));
    if (fire) sc.spk[pos] = j;
    __syncthreads();
    N2B_STAMP(a, k, 1);
    const int cnt = s_cnt;
    if (cnt == 0) return;
    if (tid == 0) {
        atomicAdd(a.counters + 1, (unsigned long long)cnt);
        atomicAdd(a.counters + 2 + P.index, (unsigned long long)cnt);
    }

    // 4. the spikes' outgoing rows
    if (n_out > 0) deliver_spikes<NPB, INL>(a, P, tile.y, CACHED ? s_cache : nullptr, cnt, n, sc, s_conn, k);
    for (int c = MERGE_OUT; c < n_out; ++c) {
        const ConnDev &C = push_at<INL>(a, P.out_first + c);
        const Row r = fire ? row_of(C, j) : Row{0, 0, 0};
        deliver_spikes_one<NPB, INL>(a, C, P.out_first + c, r, fire, pos, cnt, n, s_row, s_off, s_wsum);
    }
}

// FG items of step m's work list, one link of each per thread: every link load in flight before the reductions.
// it[0] is a listed item; it[g] is one only if g < valid (otherwise it may be anything past the list's end,
// never dereferenced: it is replaced by an empty item of connection 0 before its connection is looked up).
template <bool INL, int FG>
__device__ __forceinline__ void far_group(const StepArgs &a, const SConn *s_conn, const int4 (&it_in)[FG],
                                          const int valid, const long long m) {
    uint32_t rec[FG];
    float w[FG];
    bool h[FG];
#pragma unroll
    for (int g = 0; g < FG; ++g) {
        const int4 it = g < valid ? it_in[g] : make_int4(0, 0, 0, 0);
        const int l = it.y + (int)threadIdx.x;
        const SConn C = conn_view(a, s_conn, it.x);
        h[g] = g < valid && l < it.z;
        rec[g] = h[g] ? __ldg(C.link + l) : 0u;
        w[g] = h[g] ? link_weight(C, l) : 0.f;
    }
#pragma unroll
    for (int g = 0; g < FG; ++g)
        if (h[g]) deliver_rec(a, conn_view(a, s_conn, it_in[g].x), rec[g], w[g], m, 2);
}

// 5. the far links of step n - 1: items of NPB links, one link per thread, FG items at a time (the next
// round's items loaded under this round's links). With every block holding tiles (no tile-free blocks), the
// first ~80% of the list is split statically and, for long lists, the rest is taken in chunks of FAR_CHUNK
// rounds by whichever blocks get there first (one claim per chunk on the step's counter), so that blocks whose
// tiles ran late take less of it. With tile-free blocks, those split the whole list statically.
constexpr int FAR_CHUNK = 4;

constexpr int FAR_SPLIT_ROUNDS = 2;  // tile-free blocks take a list alone when it is at most this many rounds

// The length of step m's work list (final once step m's barrier has passed).
__device__ __forceinline__ int far_count(const StepArgs &a, const long long m) {
    return min(__ldcg(a.item_count + (int)(((m % 3) + 3) % 3)), a.item_cap);
}

template <int NPB, bool INL, int FG>
__device__ __forceinline__ void far_phase(const StepArgs &a, const long long n, const SConn *s_conn,
                                          const int count) {
    const long long m = n - 1;
    const int lst = (int)(((m % 3) + 3) % 3);
    const int4 *list = a.items + (size_t)lst * (size_t)a.item_cap;
    // the items go to the blocks without a tile when there are enough of them (a quarter of the grid) or when
    // they take them in at most FAR_SPLIT_ROUNDS rounds -- the tile blocks' step then ends with its tile --,
    // else to every block, the tile-free ones first. `count` was loaded at the step's start (under the tile's
    // loads), so every block decides alike without a load in its tile's chain.
    const int free_blocks = (int)gridDim.x - a.n_tiles;
    const bool split = free_blocks > 0 &&
                       (free_blocks >= (int)gridDim.x / 4 || count <= free_blocks * FG * FAR_SPLIT_ROUNDS);
    if (split && (int)blockIdx.x < a.n_tiles) return;
    const int G = split ? free_blocks : (int)gridDim.x;
    const int me = split ? (int)blockIdx.x - a.n_tiles : (int)blockIdx.x;
    // the first round's items loaded with the count, not after it (an item past the count is read, then ignored)
    int i = G - 1 - me;
    int4 pre[FG];
#pragma unroll
    for (int g = 0; g < FG; ++g) pre[g] = i + g * G < a.item_cap ? __ldcg(list + i + g * G) : make_int4(0, 0, 0, 0);
    // the static part: whole rounds of FG G items covering ~80% of the list; all of it for tile-free blocks and
    // for lists under 16 items per block, where the chunk claims would cost more than the imbalance
    const int stat = (split || count < 16 * G) ? count : (count * 4 / 5) / (FG * G) * (FG * G);
    for (; i < stat; i += FG * G) {
        int4 it[FG];
        int valid = 0;
#pragma unroll
        for (int g = 0; g < FG; ++g) {
            it[g] = pre[g];
            valid += i + g * G < stat;
        }
        if (i + FG * G < stat) {
#pragma unroll
            for (int g = 0; g < FG; ++g) {
                const int q = i + (FG + g) * G;
                pre[g] = q < stat ? __ldcg(list + q) : make_int4(0, 0, 0, 0);
            }
        }
        far_group<INL, FG>(a, s_conn, it, valid, m);
    }
    if (stat >= count) return;  // the same for every thread of the block
    __shared__ int s_chunk;
    int *claim = a.tile_claim + 3 + (int)(((m % 3) + 3) % 3);  // the step's chunk counter, next to the tiles'
    for (;;) {
        if (threadIdx.x == 0) s_chunk = atomicAdd(claim, 1);
        __syncthreads();
        const int c0 = stat + s_chunk * (FG * FAR_CHUNK);
        __syncthreads();  // every thread has read s_chunk before the next claim overwrites it
        if (c0 >= count) break;
        const int c1 = min(count, c0 + FG * FAR_CHUNK);
        int4 p[FG];
#pragma unroll
        for (int g = 0; g < FG; ++g) p[g] = c0 + g < c1 ? __ldcg(list + c0 + g) : make_int4(0, 0, 0, 0);
        for (int b = c0; b < c1; b += FG) {
            int4 it[FG];
#pragma unroll
            for (int g = 0; g < FG; ++g) it[g] = p[g];
            const int valid = min(FG, c1 - b);
            if (b + FG < c1) {
#pragma unroll
                for (int g = 0; g < FG; ++g) p[g] = b + FG + g < c1 ? __ldcg(list + b + FG + g) : make_int4(0, 0, 0, 0);
            }
            far_group<INL, FG>(a, s_conn, it, valid, m);
        }
    }
}

template <int NPB, bool INL, int FG, bool PULL = true>
__device__ __forceinline__ void step_body(const StepArgs &a, const long long n, int k, Neuron *cached,
                                          const int *s_cache, const SConn *s_conn, PullStage *stage) {
    __shared__ Scratch<NPB> sc;
    N2B_STAMP(a, k, 0);
    const int far_n = far_count(a, n - 1);  // in flight under the tile
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // step n + 1's list and tile counter, list n's chunk counter
        atomicExch(a.item_count + (int)((n + 1) % 3), 0);
        atomicExch(a.tile_claim + (int)((n + 1) % 3), 0);
        atomicExch(a.tile_claim + 3 + (int)((n + 1) % 3), 0);
        atomicExch(a.pull_claim + (int)((n + 1) % 3), 0);
    }
    // tile blockIdx.x first (a persistent launch holds it in registers); with fewer blocks than tiles, the
    // tiles past the first gridDim.x are claimed one at a time from the step's counter, so that blocks whose
    // tiles take longer (more spikes) take fewer of them. Thread 0's next claim is in flight under each tile.
    const bool dyn = (int)gridDim.x < a.n_tiles;
    int *claim = a.tile_claim + (int)(n % 3);
    int next = 0;
    if (dyn && threadIdx.x == 0) next = atomicAdd(claim, 1);
    Neuron nr;
    const int t = blockIdx.x;
    if (t < a.n_tiles) {
        if (cached != nullptr)
            tile_phase<NPB, INL, true, PULL>(a, n, tile_at<INL, NPB>(a, t), k, *cached, s_cache, sc, s_conn, stage);
        else
            tile_phase<NPB, INL, false, PULL>(a, n, tile_at<INL, NPB>(a, t), k, nr, nullptr, sc, s_conn, stage);
    }
    if (dyn) {
        __shared__ int s_tile;
        for (;;) {
            if (threadIdx.x == 0) s_tile = next;
            __syncthreads();
            const int u = (int)gridDim.x + s_tile;  // every thread reads it before the tile's first barrier
            if (u >= a.n_tiles) break;
            if (threadIdx.x == 0) next = atomicAdd(claim, 1);
            tile_phase<NPB, INL, false, PULL>(a, n, tile_at<INL, NPB>(a, u), k, nr, nullptr, sc, s_conn, stage);
        }
    }
    N2B_STAMP(a, k, 2);
    far_phase<NPB, INL, FG>(a, n, s_conn, far_n);
    N2B_STAMP(a, k, 5);
    if (PULL) pull_far_phase<NPB, INL>(a, n, stage);
    N2B_STAMP(a, k, 3);
}

// The warp's PullStage in the launch's dynamic shared memory (none without pull connections), initialised.
__device__ __forceinline__ PullStage *warp_stage(const StepArgs &a) {
    extern __shared__ __align__(128) unsigned char n2b_dyn_smem[];
    if (!a.pull_staged) return nullptr;
    PullStage *st = reinterpret_cast<PullStage *>(n2b_dyn_smem + (size_t)a.pull_stage_bytes * (threadIdx.x >> 5));
    pull_stage_init(st);
    return st;
}

// One step per launch: the launch boundary is the step's barrier.
template <int NPB, bool INL>
__global__ void __launch_bounds__(NPB, 2) step_kernel(const __grid_constant__ StepArgs a) {
    __shared__ SConn s_tab[SMEM_CONNS];
    const SConn *s_conn = fill_conns<INL>(a, s_tab, a.n_push);
    PullStage *stage = warp_stage(a);
    __syncthreads();
    step_body<NPB, INL, 2>(a, *a.step + a.offset, 0, nullptr, nullptr, s_conn, stage);
}

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void red_release_add(unsigned *p, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}


// Grid-wide barrier k (0, 1, ...) of a cooperative launch: every block adds 1 to one counter with release
// semantics (its writes before its arrival) and waits, with acquire loads, until the counter holds
// (k + 1) * gridDim.x -- the counter starts each launch at 0 (advance_kernel clears it after every launch).
// Every wait is bounded (a.bar_limit_ns, BAR_LIMIT_NS by default): a timeout sets error word 4 and the abort
// word, and the kernel winds down instead of hanging. Returns false once aborted. A wait ends in every case:
// its count is reached, another block's abort is seen, or its own time runs out (and it sets the abort word
// before it leaves, so that a block still waiting at this or a later barrier sees it).
__device__ __forceinline__ bool grid_sync(const StepArgs &a, unsigned k) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned *bar = a.barrier;
        const unsigned target = (k + 1) * gridDim.x;
        red_release_add(bar + BAR_COUNT, 1u);
        int ok = 1;
        unsigned long long t0 = 0;
        for (int spin = 0;; ++spin) {
            // acquire polls (measured: relaxed polls with one fence.acq_rel at the end cost ~0.4-0.9 us more per
            // step, the fence being the slower)
            if ((int)(ld_acquire(bar + BAR_COUNT) - target) >= 0) break;
            // the abort word every 16th poll (a load after the acquire waits for it: reading it on every poll
            // would double the poll's round trip); it is only set by a wait that gave up
            if ((spin & 15) == 15 && *(volatile unsigned *)(bar + BAR_ABORT)) { ok = 0; break; }
            if (spin == 0) t0 = globaltimer();
            else if (globaltimer() - t0 > a.bar_limit_ns) {
                atomicExch(bar + BAR_ABORT, 1u);
                atomicAdd(a.err + 4, 1);
                ok = 0;
                break;
            }
            __nanosleep(20);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// A window of n_steps steps in one cooperative launch (every block resident), steps separated by grid_sync.
// DENSE: three blocks per SM (registers capped for it; far items two at a time; no pull connections), for
// networks with more tiles than two blocks per SM hold -- every tile then keeps a block of its own; otherwise
// two blocks per SM and far items four at a time.
template <int NPB, bool INL, bool DENSE>
__global__ void __launch_bounds__(NPB, DENSE ? 3 : 2)
    persistent_kernel(const __grid_constant__ StepArgs a, const int n_steps) {
    if (*(volatile unsigned *)(a.barrier + BAR_ABORT)) return;  // an earlier window gave up: nothing runs
    const long long n0 = *a.step;
    // the block's first tile stays in registers for the whole window
    const bool has_tile = (int)blockIdx.x < a.n_tiles;
    const int4 tile = has_tile ? tile_at<INL, NPB>(a, blockIdx.x) : make_int4(0, 0, 0, 0);
    const PopDev &P = pop_at<INL>(a, tile.x);
    const int j = tile.y + (int)threadIdx.x;
    const bool live = has_tile && (int)threadIdx.x < tile.z;
    Neuron mine;
    load_neuron(P, j, live, mine);
    __shared__ int s_cache[3 * MERGE_OUT * NPB];
    cache_rows<NPB, INL>(a, P, j, live, s_cache);
    __shared__ SConn s_tab[SMEM_CONNS];
    const SConn *s_conn = fill_conns<INL>(a, s_tab, a.n_push);
    PullStage *stage = warp_stage(a);
    __syncthreads();
    for (int k = 0; k < n_steps; ++k) {
        step_body<NPB, INL, DENSE ? 2 : 4, !DENSE>(a, n0 + k, k, &mine, s_cache, s_conn, stage);
        if (!grid_sync(a, (unsigned)k)) break;
        N2B_STAMP(a, k, 4);
    }
    store_neuron(P, j, live, mine);
}

// After every launch: the step counter advanced, the persistent barrier's arrivals cleared.
__global__ void advance_kernel(long long *step, long long by, unsigned *barrier) {
    *step += by;
    barrier[BAR_COUNT] = 0;
}
__global__ void set_kernel(long long *p, long long value) { *p = value; }
__global__ void zero_kernel(int32_t *err, int n_err, unsigned long long *counters, int n_counters) {
    for (int k = threadIdx.x; k < n_err; k += blockDim.x) err[k] = 0;
    for (int k = threadIdx.x; k < n_counters; k += blockDim.x) counters[k] = 0;
}
__global__ void set_step_kernel(long long *step, long long value, int32_t *item_count) {
    *step = value;
    for (int k = 0; k < 12; ++k) item_count[k] = 0;  // list lengths, tile, far-chunk and pull-item counters
}

}  // namespace n2b
