// Device side of the fixed-dt hot path: Philox draws, the built-in neuron
// models, pull intake, and the fused step kernel (update -> spike ring ->
// push delivery). Written for sm_100a; included by naer2b.cu.
//
// Layout of one step of one block (a tile of NPB neurons of one population):
//   1. intake: each neuron's due arrival slot acc[n mod D][j] (int64 fixed
//      point, read and cleared), plus every pull connection's gather of its
//      incoming links against the source's spike-bit ring, plus the external
//      Poisson events -- all one exact integer sum, converted to float once;
//   2. the model's update and send (one thread per neuron);
//   3. spike-ring write: one __ballot_sync word per warp into the bit ring
//      (and the raster), the warp's spikes compacted with __popc into the
//      block's shared spike list;
//   4. push delivery: the block walks the outgoing CSR rows of its own
//      spikes as one flat (spike, link) range and adds each link's weight
//      into the target's arrival slot (n + delay) mod D with a 64-bit
//      red.global.add -- exact and order-free, so any interleaving of the
//      blocks gives the same sums.
// The next step's kernel starts after this one ends (stream order): every
// arrival of delay >= 1 is in place before it is read.
#pragma once
#include <stdint.h>

namespace n2b {

constexpr unsigned FULL = 0xffffffffu;

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
};

struct alignas(16) ConnDev {
    int32_t homogeneous, src_n, tgt_n, tgt_acc_mask;
    int32_t src_bit_mask, src_words, pad0, pad1;
    long long wfx;        // homogeneous weight, fixed point of the target
    float wscale;         // 2^shift of the target (exact)
    float pad2;
    const int32_t *ptr;
    const uint32_t *link;
    const float *w;
    long long *tgt_acc;
    const uint32_t *src_bits;
};

struct StepArgs {
    const PopDev *pops;
    const ConnDev *push;   // push connections, grouped by source population
    const ConnDev *pull;   // pull connections, grouped by target population
    const int4 *tiles;     // per block: population, first neuron, neurons
    const long long *step; // the step counter (advanced after every window)
    const long long *rec0; // raster row 0's step
    int32_t *err;
    unsigned long long *counters;
    int32_t offset;        // this launch's step = *step + offset
};

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

// Poisson count by inversion against the population's uint32 CDF table.
__device__ __forceinline__ int poisson_count(const uint32_t *__restrict__ table, int len, uint32_t u) {
    int k = 0;
    while (k < len - 1 && u >= __ldg(table + k)) ++k;
    return k;
}

__device__ __forceinline__ long long weight_fx(float w, float wscale) {
    return __float2ll_rn(__fmul_rn(w, wscale));  // exact scale, nearest-even
}

// ------------------------------------------------------------------ warp helpers

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

// ------------------------------------------------------------------ models

// Brunel's time-driven LIF (tools/brunel_reference.py:36-42 of the reference):
// refractory neurons keep V and drop their input; otherwise V = V*decay + in,
// fire at V >= theta, reset, refractory for ref_steps.
__device__ __forceinline__ bool lif_delta(const PopDev &P, int j, float in) {
    int ref = P.ref[j];
    if (ref > 0) {
        P.ref[j] = ref - 1;
        return false;
    }
    float v = __fadd_rn(__fmul_rn(P.v[j], P.p[0]), in);
    const bool fire = v >= P.p[1];
    if (fire) {
        v = P.p[2];
        P.ref[j] = P.ref_steps;
    }
    P.v[j] = v;
    return fire;
}

// PD14's LIF with exponential current synapses at fixed dt (reference
// test/networks/PD14/neuron.py:166-186): receive adds into the current, the
// exact propagators advance V and the current, threshold V > V_thresh.
__device__ __forceinline__ bool pd14(const PopDev &P, int j, float in) {
    float cur = __fadd_rn(P.i[j], in);
    float v;
    const int ref = P.ref[j];
    if (ref > 0) {
        P.ref[j] = ref - 1;
        v = P.p[5];
    } else {
        const float a = __fmul_rn(P.p[0], __fsub_rn(P.v[j], P.p[3]));
        v = __fadd_rn(__fadd_rn(P.p[3], a), __fmul_rn(P.p[2], cur));
    }
    cur = __fmul_rn(P.p[1], cur);
    const bool fire = v > P.p[4];
    if (fire) {
        v = P.p[5];
        P.ref[j] = P.ref_steps;
    }
    P.v[j] = v;
    P.i[j] = cur;
    return fire;
}

// ------------------------------------------------------------------ pull intake

// Every pull connection into the population: each warp walks the incoming
// rows of its 32 neurons one after another, the lanes striding a row
// (coalesced link loads), testing each link's source bit in the ring row of
// step n - delay; the warp's sum lands in the row's owner lane.
__device__ __forceinline__ long long pull_intake(const StepArgs &a, const PopDev &P, int first, int count,
                                                 long long n) {
    const int lane = threadIdx.x & 31;
    const int wbase = first + (threadIdx.x & ~31);
    const int nq = min(32, first + count - wbase);
    long long mine = 0;
    for (int c = P.pull_first; c < P.pull_first + P.n_pull; ++c) {
        const ConnDev C = a.pull[c];
        for (int q = 0; q < nq; ++q) {
            const int jq = wbase + q;
            const int r0 = __ldg(C.ptr + jq), r1 = __ldg(C.ptr + jq + 1);
            long long part = 0;
            for (int l = r0 + lane; l < r1; l += 32) {
                const uint32_t rec = __ldg(C.link + l);
                const int d = (int)(rec >> 24), s = (int)(rec & 0xFFFFFFu);
                if (d >= 1 && d <= C.src_bit_mask && s < C.src_n) {
                    const uint32_t word =
                        __ldg(C.src_bits + (size_t)((n - d) & C.src_bit_mask) * C.src_words + (s >> 5));
                    if ((word >> (s & 31)) & 1u)
                        part += C.homogeneous ? C.wfx : weight_fx(__ldg(C.w + l), C.wscale);
                } else {
                    atomicAdd(a.err + 1, 1);
                }
            }
            part = warp_sum64(part);
            if (lane == q) mine += part;
        }
    }
    return mine;
}

// ------------------------------------------------------------------ the step kernel

template <int NPB>
__global__ void __launch_bounds__(NPB) step_kernel(const StepArgs a) {
    constexpr int NW = NPB / 32;
    __shared__ int s_cnt;
    __shared__ int s_spk[NPB];
    __shared__ int s_row[NPB];
    __shared__ int s_off[NPB + 1];
    __shared__ int s_wsum[NW];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int4 tile = a.tiles[blockIdx.x];
    const PopDev P = a.pops[tile.x];  // a register copy: the state stores cannot alias it
    const long long n = *a.step + a.offset;
    const int j = tile.y + tid;
    const bool live = tid < tile.z;
    if (tid == 0) s_cnt = 0;

    // 1-2. intake and update
    bool fire = false;
    const int model = P.model;
    if (model == 3) {  // N2B_MODEL_POISSON_SOURCE
        fire = live && draw(P, j, n, 1u) < P.fire_threshold;
    } else {
        long long acc = 0;
        if (live) {
            long long *slot = P.acc + (size_t)(n & P.acc_mask) * (size_t)P.n + j;
            acc = *slot;
            *slot = 0;
        }
        if (P.n_pull > 0) acc += pull_intake(a, P, tile.y, tile.z, n);
        if (live) {
            if (P.ext_len > 0) acc += (long long)poisson_count(P.ext_table, P.ext_len, draw(P, j, n, 0u)) * P.ext_wfx;
            const float in = __fmul_rn(__ll2float_rn(acc), P.inv_scale);
            fire = (model == 1) ? lif_delta(P, j, in) : pd14(P, j, in);
        }
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
    if (fire) s_spk[base + __popc(b & ((1u << lane) - 1u))] = j;
    __syncthreads();
    const int cnt = s_cnt;
    if (cnt == 0) return;
    if (tid == 0) {
        atomicAdd(a.counters + 1, (unsigned long long)cnt);
        atomicAdd(a.counters + 2 + P.index, (unsigned long long)cnt);
    }

    // 4. push delivery of the block's spikes, one flat (spike, link) range per connection
    for (int c = P.out_first; c < P.out_first + P.n_out; ++c) {
        const ConnDev C = a.push[c];
        int deg = 0;
        if (tid < cnt) {
            const int s = s_spk[tid];
            const int r0 = __ldg(C.ptr + s);
            deg = __ldg(C.ptr + s + 1) - r0;
            s_row[tid] = r0;
        }
        const int incl = warp_incl_scan(deg);
        if (lane == 31) s_wsum[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int v = lane < NW ? s_wsum[lane] : 0;
            v = warp_incl_scan(v);
            if (lane < NW) s_wsum[lane] = v;
        }
        __syncthreads();
        if (tid < cnt) s_off[tid] = incl - deg + (warp > 0 ? s_wsum[warp - 1] : 0);
        if (tid == 0) s_off[cnt] = s_wsum[NW - 1];
        __syncthreads();
        const int total = s_off[cnt];
        const size_t tn = (size_t)C.tgt_n;
        for (int idx = tid; idx < total; idx += NPB) {
            int lo = 0, hi = cnt;  // s_off[lo] <= idx < s_off[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (s_off[mid] <= idx) lo = mid; else hi = mid;
            }
            const int l = s_row[lo] + (idx - s_off[lo]);
            const uint32_t rec = __ldg(C.link + l);
            const int d = (int)(rec >> 24), t = (int)(rec & 0xFFFFFFu);
            const long long wfx = C.homogeneous ? C.wfx : weight_fx(__ldg(C.w + l), C.wscale);
            if (d >= 1 && d <= C.tgt_acc_mask && t < C.tgt_n) {
                atomicAdd(reinterpret_cast<unsigned long long *>(C.tgt_acc + (size_t)((n + d) & C.tgt_acc_mask) * tn + t),
                          (unsigned long long)wfx);
            } else {
                atomicAdd(a.err + 0, 1);
            }
        }
        if (tid == 0) atomicAdd(a.counters + 0, (unsigned long long)total);
        __syncthreads();
    }
}

__global__ void advance_kernel(long long *step, long long by) { *step += by; }
__global__ void set_kernel(long long *p, long long value) { *p = value; }
__global__ void zero_kernel(int32_t *err, int n_err, unsigned long long *counters, int n_counters) {
    for (int k = threadIdx.x; k < n_err; k += blockDim.x) err[k] = 0;
    for (int k = threadIdx.x; k < n_counters; k += blockDim.x) counters[k] = 0;
}

}  // namespace n2b
