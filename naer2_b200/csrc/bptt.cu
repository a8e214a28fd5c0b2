// Surrogate-gradient BPTT of a recurrent LIF layer with delayed sparse recurrence (include/naer2b.h,
// n2b_bptt_*). No counterpart in the reference: naer2 has no differentiable path.
//
// Model, per sample b, hidden neuron i, step t (dt = 1 step):
//   R[t][i]     = sum over incoming links k of i: w_k * s[t - d_k][pre_k]          (d_k in 1..5 steps)
//   Vpre[t][i]  = alpha * V[t-1][i] + U[t][i] + R[t][i]                             (U: input current)
//   s[t][i]     = Vpre >= theta  (spiking)   |   f(Vpre - theta), f(x) = x / (1 + slope |x|)  (smooth)
//   V[t][i]     = Vpre - theta * s[t][i]                                            (subtractive reset)
//   O[t][r]     = beta * O[t-1][r] + sum_i w_out[i][r] * s[t][i];   m[r] = max_t O[t][r] at t*[r]
// Backward (q = dL/dVpre, g = f'(Vpre - theta) = 1 / (1 + slope |Vpre - theta|)^2, the fast-sigmoid
// surrogate in the spiking model, the true derivative in the smooth one; the reset is differentiated):
//   o[t][r]  = dm[r] * [t == t*[r]] + beta * o[t+1][r]
//   q[t][i]  = alpha q[t+1][i] + g[t][i] * (sum_{k out of i} w_k q[t + d_k][post_k]
//                                           + sum_r w_out[i][r] o[t][r] - theta alpha q[t+1][i])
//   dU[t][i] = q[t][i];  dw_k = sum_t,b s[t - d_k][pre_k] q[t][post_k];  dw_out[i][r] = sum_t,b s[t][i] o[t][r]
//
// Layout: a group of 8 CTAs runs 8 samples; CTA `rank` owns hidden neurons [rank*HC, rank*HC + HC), HC = H/8,
// four threads per neuron (two samples each; the link loops split a row among the four, interleaved). The
// forward's group is a thread-block cluster; the adjoint's is a plain group of one cooperative launch (one
// CTA per SM: at that size only 15 clusters of 8 are resident on 148 SMs, but every group must be).
// Forward: every CTA keeps the spikes of the last 6 steps of all H neurons for its 8 samples (one byte of 8
// sample bits per neuron, or 8 floats in the smooth model) in shared memory; each step a neuron's new entry
// is written into all 8 CTAs' rings (distributed shared memory) before one cluster barrier. Backward: each
// K-step segment is first recomputed from its membrane checkpoint and the stored spikes of every step by two
// grid-wide kernels (the recurrent inputs of all its steps at once, then one membrane scan per neuron and
// sample; same arithmetic, same order: the same Vpre bit for bit), then run backwards by one
// cooperative launch; q of all neurons is exchanged through a two-slot ring in global memory (L2) with one
// counted arrival per CTA and step, and each neuron pushes its outgoing rows' q sums into a 6-slot ring of its
// own partials, kept in global memory between the segments' launches.
// Every sum has a fixed order (no float atomics), so results are bit-for-bit reproducible.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/naer2b.h"

namespace cg = cooperative_groups;

namespace n2b_bptt {

constexpr int NS = 8;          // samples per cluster
constexpr int CL = 8;          // CTAs per cluster
constexpr int NT = 4;          // threads per neuron
constexpr int SPT = NS / NT;   // samples per thread
constexpr int RING = 6;        // spike / partial ring slots (delays 1..5)
constexpr int MAXD = 5;
constexpr unsigned FULL = 0xffffffffu;

struct Args {
    int B, T, H, R, K, HC, NC, nseg, nnz;
    float alpha, beta, theta, slope;
    int tape, csr_smem;
    const int32_t *in_ptr;
    const uint16_t *in_code;
    const float *in_w;
    const int32_t *out_grp;  // [H][MAXD + 1]: row start of each delay 1..5, then the row end
    const uint16_t *out_code;
    const float *out_w;
    const float *U;     // [T][B][H]
    uint8_t *s_bits;    // [T][NC][H]      (spiking)
    float *s_f;         // [T][NC][H][8]   (smooth)
    float *v_ckpt;      // [nseg][B][H]
    float *g_seg;       // [K][B][H]: the segment's recurrent input, then its surrogate derivatives
    float *dU;          // [T][B][H]
    const float *w_out; // [H][R]
    float *m;           // [B][R]
    int32_t *tstar;     // [B][R]
    const float *dm;    // [B][R]
    const int32_t *tstar_in;
    float *dwp;         // [NC][nnz] per-cluster dw, out order
    float *dwo_p;       // [NC][H][R]
    float *part_st;     // [NC * CL][RING][HC][NS] the adjoint's partial ring between segments
    float *q_st;        // [B][H] q[t0] of the last segment done
    float *o_st;        // [B][R] the readout adjoint at t0
    float *qx;          // [NC][2][H][8] the adjoint's q exchange ring (slot t & 1)
    uint32_t *xcnt;     // [NC] the adjoint's arrivals per group (zeroed before each launch)
    int32_t *err;       // [N2B_BPTT_ERR_WORDS]
    int wait_polls;     // polls before an exchange wait gives up
};

__device__ __forceinline__ float surrogate(float x, float slope) {
    const float a = __fadd_rn(1.f, __fmul_rn(slope, fabsf(x)));
    return __fdiv_rn(1.f, __fmul_rn(a, a));
}

__device__ __forceinline__ float smooth_spike(float x, float slope) {
    return __fdiv_rn(x, __fadd_rn(1.f, __fmul_rn(slope, fabsf(x))));
}

// v[k] of a thread's two samples: (sub's samples 2 sub, 2 sub + 1) with compile-time indices only.
__device__ __forceinline__ void mine(const float v[NS], int sub, float &x0, float &x1) {
    x0 = sub == 0 ? v[0] : sub == 1 ? v[2] : sub == 2 ? v[4] : v[6];
    x1 = sub == 0 ? v[1] : sub == 1 ? v[3] : sub == 2 ? v[5] : v[7];
}

// Shared-memory layout of the forward kernel (identical in every CTA, so that remote addresses match).
struct FwdSmem {
    size_t ring, xbuf, wout, ptr, code, w, total;
};
__host__ __device__ inline FwdSmem fwd_smem(int H, int HC, int R, bool smooth, bool csr_smem, int in_cta_max) {
    FwdSmem L{};
    size_t o = 0;
    auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
    L.ring = o; o = a16(o + (smooth ? sizeof(float) * RING * H * NS : (size_t)RING * H));
    L.xbuf = o; o = a16(o + sizeof(float) * 2 * CL * NS * R);
    L.wout = o; o = a16(o + sizeof(float) * HC * R);
    L.ptr = o; o = a16(o + sizeof(int32_t) * (HC + 1));
    L.code = o; o = a16(o + (csr_smem ? sizeof(uint16_t) * in_cta_max : 0));
    L.w = o; o = a16(o + (csr_smem ? sizeof(float) * in_cta_max : 0));
    L.total = o;
    return L;
}

constexpr int QROW = 12;  // floats per neuron in the q exchange buffer: 8 samples, padded for the banks

struct BwdSmem {
    size_t pnew, part, dwo, obuf, grp, code, w, dw, total;
};
__host__ __device__ inline BwdSmem bwd_smem(int H, int HC, int R, int out_cta_max) {
    BwdSmem L{};
    size_t o = 0;
    auto a16 = [](size_t x) { return (x + 15) & ~size_t(15); };
    L.pnew = o; o = a16(o + sizeof(float) * H * QROW);
    L.part = o; o = a16(o + sizeof(float) * RING * HC * NS);
    L.dwo = o; o = a16(o + sizeof(float) * HC * R);
    L.obuf = o; o = a16(o + sizeof(float) * 2 * NS * R);  // o[t] in half t & 1
    L.grp = o; o = a16(o + sizeof(int32_t) * HC * (MAXD + 1));
    L.code = o; o = a16(o + sizeof(uint16_t) * out_cta_max);
    L.w = o; o = a16(o + sizeof(float) * out_cta_max);
    L.dw = o; o = a16(o + sizeof(float) * out_cta_max);
    L.total = o;
    return L;
}

// One CTA's arrival at a group step (thread 0, after a __syncthreads that follows the CTA's writes): a release
// add on the group's counter; later (other work in between), a bounded acquire spin until `target` arrivals
// (every CTA of the group at this step). A wait that gives up counts in err[3] and sets `aborted`, after which
// the CTA still arrives but no longer waits, so that neither it nor the CTAs that wait for its arrivals can hang.
constexpr int XCHG_SPIN_LIMIT = 1 << 21;  // default polls (n2b_bptt_desc.wait_polls = 0): about a second
__device__ __forceinline__ void group_arrive(uint32_t *cnt) {
    __threadfence();
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
}
__device__ __forceinline__ void group_wait(const uint32_t *cnt, uint32_t target, int32_t *err, int limit,
                                           int &aborted) {
    if (aborted) return;
    for (int it = 0;; ++it) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(cnt) : "memory");
        if (v >= target) return;
        if (it >= limit) {
            atomicAdd(err + 3, 1);
            aborted = 1;
            return;
        }
    }
}

// The spikes that the incoming links read: the forward's shared-memory ring (6 slots, the slot of step t in
// t mod 6; slots of steps before 0 are still zero), or the stored spikes of every step (recompute).
struct RingSrc {
    const unsigned char *ring;
    int H, tbase;  // t mod 6
    __device__ __forceinline__ int slot(int d) const {
        const int sl = tbase - d;
        return sl < 0 ? sl + RING : sl;
    }
};
struct TapeSrc {
    const uint8_t *bits;
    const float *f;
    int H, NC, q, t;
};

// R for the 8 samples of one neuron: this thread's share of its incoming row (links rs + sub, rs + sub + NT,
// ...), then the NT shares added pairwise ((s0 + s1) + (s2 + s3), the same value in all NT lanes).
// CHECKED: every code is checked (a bad one counted and skipped); otherwise the rows were validated when they
// were copied (bad links replaced by a zero-weight link). Both give the same sums for the same rows.
template <bool SMOOTH, bool CHECKED, class Src>
__device__ __forceinline__ void gather_in(const Args &a, const Src &src, const uint16_t *code, const float *w,
                                          int rs, int re, int sub, float acc[NS]) {
#pragma unroll
    for (int b = 0; b < NS; ++b) acc[b] = 0.f;
#pragma unroll 2
    for (int l = rs + sub; l < re; l += NT) {
        const uint32_t c = code[l];
        const float wl = w[l];
        const int pre = (int)(c & 0x7FFu), d = (int)(c >> 11);
        if (CHECKED && (d < 1 || d > MAXD || pre >= a.H)) {
            atomicAdd(a.err + 0, 1);
            continue;
        }
        if constexpr (SMOOTH) {
            float s[NS];
            if constexpr (std::is_same<Src, RingSrc>::value) {
                const float4 *p = reinterpret_cast<const float4 *>(src.ring) + ((size_t)src.slot(d) * src.H + pre) * 2;
                const float4 x = p[0], y = p[1];
                s[0] = x.x; s[1] = x.y; s[2] = x.z; s[3] = x.w; s[4] = y.x; s[5] = y.y; s[6] = y.z; s[7] = y.w;
            } else {
                const int tt = src.t - d;
                if (tt < 0) continue;
                const float4 *p = reinterpret_cast<const float4 *>(src.f) + (((size_t)tt * src.NC + src.q) * src.H + pre) * 2;
                const float4 x = p[0], y = p[1];
                s[0] = x.x; s[1] = x.y; s[2] = x.z; s[3] = x.w; s[4] = y.x; s[5] = y.y; s[6] = y.z; s[7] = y.w;
            }
#pragma unroll
            for (int b = 0; b < NS; ++b) acc[b] = __fadd_rn(acc[b], __fmul_rn(wl, s[b]));
        } else {
            uint32_t byte;
            if constexpr (std::is_same<Src, RingSrc>::value) {
                byte = src.ring[(size_t)src.slot(d) * src.H + pre];
            } else {
                const int tt = src.t - d;
                byte = tt >= 0 ? src.bits[((size_t)tt * src.NC + src.q) * src.H + pre] : 0u;
            }
            if (!byte) continue;
#pragma unroll
            for (int b = 0; b < NS; ++b)
                if ((byte >> b) & 1u) acc[b] = __fadd_rn(acc[b], wl);
        }
    }
#pragma unroll
    for (int b = 0; b < NS; ++b) acc[b] = __fadd_rn(acc[b], __shfl_xor_sync(FULL, acc[b], 1));
#pragma unroll
    for (int b = 0; b < NS; ++b) acc[b] = __fadd_rn(acc[b], __shfl_xor_sync(FULL, acc[b], 2));
}

// One membrane step of one sample: returns the spike value, updates V, gives Vpre.
template <bool SMOOTH>
__device__ __forceinline__ float lif_step(const Args &a, float &V, float u, float r, float &vpre) {
    const float vp = __fadd_rn(__fadd_rn(__fmul_rn(a.alpha, V), u), r);
    float s;
    if constexpr (SMOOTH) s = smooth_spike(__fadd_rn(vp, -a.theta), a.slope);
    else s = vp >= a.theta ? 1.f : 0.f;
    V = __fadd_rn(vp, -__fmul_rn(a.theta, s));
    vpre = vp;
    return s;
}

// ------------------------------------------------------------------------------------------------ forward

template <bool SMOOTH>
__global__ void __launch_bounds__(512) fwd_kernel(const __grid_constant__ Args a, int in_cta_max) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int q = (int)blockIdx.x / CL;
    const int H = a.H, HC = a.HC, R = a.R, B = a.B;
    const int h0 = rank * HC;
    const bool csr = a.csr_smem != 0;
    const FwdSmem L = fwd_smem(H, HC, R, SMOOTH, csr, in_cta_max);
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *ring = smem + L.ring;
    float *xbuf = reinterpret_cast<float *>(smem + L.xbuf);
    float *wout = reinterpret_cast<float *>(smem + L.wout);
    int32_t *lptr = reinterpret_cast<int32_t *>(smem + L.ptr);
    const int tid = threadIdx.x, nthr = blockDim.x;

    for (size_t k = tid; k < (L.xbuf - L.ring) / 4; k += nthr) reinterpret_cast<uint32_t *>(ring)[k] = 0u;
    for (int k = tid; k < HC * R; k += nthr) wout[k] = a.w_out[(size_t)h0 * R + k];
    const int base = a.in_ptr[h0];
    for (int k = tid; k <= HC; k += nthr) lptr[k] = a.in_ptr[h0 + k] - base;
    const uint16_t *gcode = a.in_code + base;
    const float *gw = a.in_w + base;
    const int n_in = a.in_ptr[h0 + HC] - base;
    const bool in_smem = csr && n_in <= in_cta_max;
    if (csr && !in_smem && tid == 0) atomicAdd(a.err + 2, 1);  // a wrong in_cta_max: the rows stay global
    uint16_t *sc = reinterpret_cast<uint16_t *>(smem + L.code);
    float *sw = reinterpret_cast<float *>(smem + L.w);
    if (in_smem) {
        for (int k = tid; k < n_in; k += nthr) {  // validated once: a bad link becomes a zero-weight link
            const uint32_t c = gcode[k];
            const bool bad = (c >> 11) < 1 || (c >> 11) > MAXD || (c & 0x7FFu) >= (uint32_t)H;
            if (bad) atomicAdd(a.err + 0, 1);
            sc[k] = bad ? (uint16_t)(1u << 11) : (uint16_t)c;
            sw[k] = bad ? 0.f : gw[k];
        }
    }
    __syncthreads();
    cl.sync();  // every CTA's shared memory is initialised before any remote write reaches it

    const bool nt = tid < NT * HC;
    const int pl = nt ? tid / NT : 0, sub = tid % NT;
    const int post = h0 + pl;
    const int rs = nt ? lptr[pl] : 0, re = nt ? lptr[pl + 1] : 0;
    float V0 = 0.f, V1 = 0.f;
    const bool ro = tid < NS * R;
    const int rb = ro ? tid / R : 0, rr = ro ? tid % R : 0;
    float O = 0.f, mx = -INFINITY;
    int ts = -1;
    const size_t bq = (size_t)q * NS + SPT * sub;  // this thread's first sample

    for (int t = 0; t < a.T; ++t) {
        if (a.tape && t % a.K == 0 && nt) {
            a.v_ckpt[((size_t)(t / a.K) * B + bq) * H + post] = V0;
            a.v_ckpt[((size_t)(t / a.K) * B + bq + 1) * H + post] = V1;
        }
        float acc[NS];
        const RingSrc src{ring, H, t % RING};
        if (in_smem) gather_in<SMOOTH, false>(a, src, sc, sw, rs, re, sub, acc);
        else gather_in<SMOOTH, true>(a, src, gcode, gw, rs, re, sub, acc);
        float r0, r1, s0 = 0.f, s1 = 0.f, vp;
        mine(acc, sub, r0, r1);
        if (nt) {
            const float u0 = __ldg(a.U + ((size_t)t * B + bq) * H + post);
            const float u1 = __ldg(a.U + ((size_t)t * B + bq + 1) * H + post);
            s0 = lif_step<SMOOTH>(a, V0, u0, r0, vp);
            s1 = lif_step<SMOOTH>(a, V1, u1, r1, vp);
        }
        const int slot = t % RING;
        if constexpr (SMOOTH) {
            if (nt) {
                const float2 v = make_float2(s0, s1);
                float2 *dst = reinterpret_cast<float2 *>(ring) + ((size_t)slot * H + post) * 4 + sub;
                for (int k = 0; k < CL; ++k) *cl.map_shared_rank(dst, k) = v;
                if (a.tape) reinterpret_cast<float2 *>(a.s_f)[(((size_t)t * a.NC + q) * H + post) * 4 + sub] = v;
            }
        } else {
            uint32_t bits = ((s0 != 0.f) ? 1u : 0u) | ((s1 != 0.f) ? 2u : 0u);
            bits <<= SPT * sub;
            bits |= __shfl_xor_sync(FULL, bits, 1);
            bits |= __shfl_xor_sync(FULL, bits, 2);
            if (nt) {
                unsigned char *dst = ring + (size_t)slot * H + post;
                for (int k = sub; k < CL; k += NT) *cl.map_shared_rank(dst, k) = (unsigned char)bits;
                if (a.tape && sub == 0) a.s_bits[((size_t)t * a.NC + q) * H + post] = (uint8_t)bits;
            }
        }
        __syncthreads();  // this CTA's own neurons' entries are in its ring
        if (ro) {
            float sum = 0.f;
            if constexpr (SMOOTH) {
                const float *rf = reinterpret_cast<const float *>(ring) + ((size_t)slot * H + h0) * NS + rb;
                for (int p = 0; p < HC; ++p) sum = __fadd_rn(sum, __fmul_rn(rf[(size_t)p * NS], wout[p * R + rr]));
            } else {  // four neurons' bytes per word, neurons in ascending order
                const uint32_t *rw = reinterpret_cast<const uint32_t *>(ring + (size_t)slot * H + h0);
                for (int k = 0; k < HC / 4; ++k) {
                    const uint32_t word = rw[k];
                    if (!word) continue;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if ((word >> (8 * j + rb)) & 1u) sum = __fadd_rn(sum, wout[(4 * k + j) * R + rr]);
                }
            }
            float *dst = xbuf + (((size_t)(t & 1) * CL + rank) * NS + rb) * R + rr;
            *cl.map_shared_rank(dst, 0) = sum;
        }
        cl.sync();  // step t's spikes in every ring, its readout partials in rank 0
        if (rank == 0 && ro) {
            float tot = 0.f;
            for (int k = 0; k < CL; ++k) tot = __fadd_rn(tot, xbuf[(((size_t)(t & 1) * CL + k) * NS + rb) * R + rr]);
            O = __fadd_rn(__fmul_rn(a.beta, O), tot);
            if (O > mx) {
                mx = O;
                ts = t;
            }
        }
    }
    if (rank == 0 && ro) {
        a.m[(size_t)(q * NS + rb) * R + rr] = mx;
        a.tstar[(size_t)(q * NS + rb) * R + rr] = ts;
    }
    cl.sync();  // no CTA leaves while another may still address its shared memory
}

// ------------------------------------------------------------------------------------------------ recompute

// The recurrent input R of every step of a segment [t0, t1) from the stored spikes: NT threads per
// (chunk of TC steps, cluster, neuron); each thread decodes its share of the neuron's incoming row once and
// applies every link to the TC steps of its chunk, then the NT shares are added as the forward adds them
// ((s0 + s1) + (s2 + s3), links in the forward's order within each share): the same sums bit for bit.
// A link with a bad code (counted by the forward) is clamped into range here instead of checked per step.
// Spiking model: a block is blockDim / NT neurons of one (chunk, cluster); it first stages the spike bytes of
// the MAXD + TC - 1 steps its links read, of every neuron of the cluster, as one 16-byte row per neuron in
// shared memory (steps before 0 as zero), so that a link's TC steps are one 128-bit load. Launch: grid
// (H / (blockDim / NT), NC, chunks).
constexpr int TC = 5;
constexpr int RWIN = MAXD + TC - 1;  // steps tc - MAXD .. tc + TC - 2
static_assert(RWIN <= 16, "a staged row is 16 bytes");

template <bool SMOOTH>
__global__ void __launch_bounds__(256) recompute_r_kernel(const __grid_constant__ Args a, int t0, int t1) {
    extern __shared__ __align__(16) unsigned char rows[];  // spiking: [H][16] bytes
    const int ppb = blockDim.x / NT;  // neurons per block
    const int q = blockIdx.y, tc = t0 + blockIdx.z * TC;
    const int post = blockIdx.x * ppb + threadIdx.x / NT, sub = threadIdx.x % NT;
    const int rs = a.in_ptr[post], re = a.in_ptr[post + 1];
    const int kend = min(TC, t1 - tc);  // steps of this chunk inside the segment
    float acc[TC][NS];
#pragma unroll
    for (int k = 0; k < TC; ++k)
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[k][b] = 0.f;
    if constexpr (SMOOTH) {
        const int row = a.NC * a.H;  // entries between two steps of the stored spikes
        for (int l = rs + sub; l < re; l += NT) {
            const uint32_t c = a.in_code[l];
            const float wl = a.in_w[l];
            const int pre = min((int)(c & 0x7FFu), a.H - 1), d = min(max((int)(c >> 11), 1), MAXD);
            const int base = (tc - d) * row + q * a.H + pre;  // step tc - d
#pragma unroll
            for (int k = 0; k < TC; ++k) {
                if (tc + k - d < 0 || k >= kend) continue;
                const float4 *p = reinterpret_cast<const float4 *>(a.s_f) + (size_t)(base + k * row) * 2;
                const float4 x = p[0], y = p[1];
                const float sv[NS] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
#pragma unroll
                for (int b = 0; b < NS; ++b) acc[k][b] = __fadd_rn(acc[k][b], __fmul_rn(wl, sv[b]));
            }
        }
    } else {
        // stage: thread j packs the RWIN bytes of neurons j, j + blockDim, ... (coalesced byte loads per step)
        for (int pre = threadIdx.x; pre < a.H; pre += blockDim.x) {
            uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int sidx = 0; sidx < RWIN; ++sidx) {
                const int tt = tc - MAXD + sidx;
                const uint32_t byte = (tt >= 0 && tt < a.T) ? a.s_bits[((size_t)tt * a.NC + q) * a.H + pre] : 0u;
                w[sidx / 4] |= byte << (8 * (sidx % 4));
            }
            reinterpret_cast<uint4 *>(rows)[pre] = make_uint4(w[0], w[1], w[2], w[3]);
        }
        __syncthreads();
        for (int l = rs + sub; l < re; l += NT) {
            const uint32_t c = a.in_code[l];
            const float wl = a.in_w[l];
            const int pre = min((int)(c & 0x7FFu), a.H - 1), d = min(max((int)(c >> 11), 1), MAXD);
            const uint4 v = reinterpret_cast<const uint4 *>(rows)[pre];
            const uint64_t lo = ((uint64_t)v.y << 32) | v.x, hi = ((uint64_t)v.w << 32) | v.z;
            const int sh = 8 * (MAXD - d);  // byte of step tc - d
            const uint64_t win = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;  // steps tc - d ...
            if (!(win & ((1ull << (8 * TC)) - 1))) continue;
            // branch-free: a clear bit adds +0.0f, which leaves a sum that started at +0 unchanged bit for bit
            // (it is never -0), so the sums stay the forward's
#pragma unroll
            for (int k = 0; k < TC; ++k) {
                const uint32_t byte = k < kend ? (uint32_t)(win >> (8 * k)) & 0xffu : 0u;
#pragma unroll
                for (int b = 0; b < NS; ++b) acc[k][b] = __fadd_rn(acc[k][b], ((byte >> b) & 1u) ? wl : 0.f);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < TC; ++k) {
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[k][b] = __fadd_rn(acc[k][b], __shfl_xor_sync(FULL, acc[k][b], 1));
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[k][b] = __fadd_rn(acc[k][b], __shfl_xor_sync(FULL, acc[k][b], 2));
    }
    const size_t bq = (size_t)q * NS + SPT * sub;
#pragma unroll
    for (int k = 0; k < TC; ++k) {
        if (k >= kend) break;
        float r0, r1;
        mine(acc[k], sub, r0, r1);
        a.g_seg[((size_t)(tc + k - t0) * a.B + bq) * a.H + post] = r0;
        a.g_seg[((size_t)(tc + k - t0) * a.B + bq + 1) * a.H + post] = r1;
    }
}

// The membrane of the segment from its checkpoint, one thread per (sample, neuron): Vpre as the forward made it,
// its surrogate derivative over R in g_seg, and a check that the stored spike is the one Vpre gives.
template <bool SMOOTH>
__global__ void __launch_bounds__(256) recompute_v_kernel(const __grid_constant__ Args a, int seg, int t0, int t1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.B * a.H) return;
    const int b = k / a.H, j = k % a.H, q = b / NS, bl = b % NS;
    float V = a.v_ckpt[(size_t)seg * a.B * a.H + k];
    int bad = 0;
    for (int t = t0; t < t1; ++t) {
        float *gp = a.g_seg + (size_t)(t - t0) * a.B * a.H + k;
        const float u = __ldg(a.U + (size_t)t * a.B * a.H + k);
        float vp;
        const float s = lif_step<SMOOTH>(a, V, u, *gp, vp);
        float stored;
        if constexpr (SMOOTH) stored = a.s_f[(((size_t)t * a.NC + q) * a.H + j) * NS + bl];
        else stored = ((a.s_bits[((size_t)t * a.NC + q) * a.H + j] >> bl) & 1u) ? 1.f : 0.f;
        bad += s != stored;
        *gp = surrogate(__fadd_rn(vp, -a.theta), a.slope);
    }
    if (bad) atomicAdd(a.err + 1, bad);  // the recompute differs from the forward
}

// ------------------------------------------------------------------------------------------------ adjoint

// One delay group of a neuron's outgoing row at step t: acc[b] += w q[t][post][b] over this thread's share
// of the links (gs + sub, gs + sub + NT, ...), OUT_U links a round: all loads of a round (codes, weights, q
// rows, dw) are issued before its arithmetic and stores, so that a round costs one chain of shared-memory
// latencies. With DW (warp-uniform: some lane's neuron spiked at t - d), the lanes with `dwl` also add
// sum_b s[b] q[t][post][b] to dw[l]. A skipped code (0xFFFF) reads row 0 and adds nothing.
constexpr int OUT_U = 4;
template <bool SMOOTH, bool DW>
__device__ __forceinline__ void out_group(const uint16_t *ocode, const float *ow, const float *pnew, float *dw,
                                          int gs, int ge, int sub, bool dwl, uint32_t sbyte, const float *sf,
                                          float acc[NS]) {
    for (int base = gs + sub; base < ge; base += OUT_U * NT) {
        uint32_t c[OUT_U];
        float wl[OUT_U], od[OUT_U];
        float4 y0[OUT_U], y1[OUT_U];
        bool ok[OUT_U];
#pragma unroll
        for (int u = 0; u < OUT_U; ++u) {
            const int l = base + u * NT;
            c[u] = l < ge ? ocode[l] : 0xFFFFu;
            wl[u] = l < ge ? ow[l] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < OUT_U; ++u) {
            ok[u] = c[u] != 0xFFFFu;
            const size_t post = ok[u] ? (c[u] & 0x7FFu) : 0u;  // < H: checked when the rows were copied
            y0[u] = reinterpret_cast<const float4 *>(pnew)[post * (QROW / 4)];
            y1[u] = reinterpret_cast<const float4 *>(pnew)[post * (QROW / 4) + 1];
            if constexpr (DW) od[u] = (dwl && ok[u]) ? dw[base + u * NT] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < OUT_U; ++u) {
            if (!ok[u]) continue;
            const float x[NS] = {y0[u].x, y0[u].y, y0[u].z, y0[u].w, y1[u].x, y1[u].y, y1[u].z, y1[u].w};
#pragma unroll
            for (int b = 0; b < NS; ++b) acc[b] = __fmaf_rn(wl[u], x[b], acc[b]);
            if constexpr (DW) {
                if (dwl) {
                    float dk = 0.f;
#pragma unroll
                    for (int b = 0; b < NS; ++b) {
                        if constexpr (SMOOTH) dk = __fmaf_rn(sf[b], x[b], dk);
                        else if ((sbyte >> b) & 1u) dk = __fadd_rn(dk, x[b]);
                    }
                    dw[base + u * NT] = __fadd_rn(od[u], dk);
                }
            }
        }
    }
}

// The adjoint of segment [t0, t1), run backwards; `first`: the last segment of the sequence (state starts at
// zero), else the state of the segment after it is loaded (partial ring, q, readout adjoint, dw, dw_out).
// Each step, every CTA writes the q[t] of its neurons into slot t & 1 of the group's ring in global memory,
// arrives on the group's counter, waits for all 8 arrivals and copies q[t] of all H neurons into its own
// shared buffer (pnew). Two slots suffice: a CTA writes slot t & 1 only after every CTA of the group arrived
// at step t + 1, which each does after its copy of slot t & 1 at step t + 2. The launch is cooperative, so
// the CTAs of a group are resident together; `g0` is the launch's first group.
template <bool SMOOTH>
__global__ void __launch_bounds__(512) bwd_kernel(const __grid_constant__ Args a, int out_cta_max, int t0, int t1,
                                                   int first, int g0) {
    const int rank = (int)blockIdx.x % CL;
    const int q = g0 + (int)blockIdx.x / CL;
    const int H = a.H, HC = a.HC, R = a.R, B = a.B;
    const int h0 = rank * HC;
    const BwdSmem L = bwd_smem(H, HC, R, out_cta_max);
    extern __shared__ __align__(16) unsigned char smem[];
    float *pnew = reinterpret_cast<float *>(smem + L.pnew);
    float *part = reinterpret_cast<float *>(smem + L.part);
    const float *wout = a.w_out + (size_t)h0 * R;  // read through L1
    float *dwo = reinterpret_cast<float *>(smem + L.dwo);
    float *obuf = reinterpret_cast<float *>(smem + L.obuf);
    int32_t *grp = reinterpret_cast<int32_t *>(smem + L.grp);
    uint16_t *ocode = reinterpret_cast<uint16_t *>(smem + L.code);
    float *ow = reinterpret_cast<float *>(smem + L.w);
    float *dw = reinterpret_cast<float *>(smem + L.dw);
    const int tid = threadIdx.x, nthr = blockDim.x;
    float *part_st = a.part_st + ((size_t)q * CL + rank) * RING * HC * NS;  // this group's CTA, in any launch

    const bool nt = tid < NT * HC;
    const int pl = nt ? tid / NT : 0, sub = tid % NT;
    const int me = h0 + pl;  // this thread's neuron (the pre of its outgoing row)
    const int obase = a.out_grp[(size_t)h0 * (MAXD + 1)];
    const int on_all = a.out_grp[(size_t)(h0 + HC - 1) * (MAXD + 1) + MAXD] - obase;
    const int on = min(on_all, out_cta_max);  // a wrong out_cta_max: the links past it are skipped, counted
    if (on_all > on && tid == 0) atomicAdd(a.err + 2, 1);
    for (size_t k = tid; k < L.total / 4; k += nthr) reinterpret_cast<uint32_t *>(smem)[k] = 0u;
    __syncthreads();
    for (int k = tid; k < HC * (MAXD + 1); k += nthr) grp[k] = min(a.out_grp[(size_t)h0 * (MAXD + 1) + k] - obase, on);
    // the outgoing rows, validated once: a link whose target is out of range or whose delay is not its group's
    // becomes the code 0xFFFF (skipped) and is counted
    if (nt) {
        for (int d = 1; d <= MAXD; ++d) {
            const int gs = min(a.out_grp[(size_t)me * (MAXD + 1) + d - 1] - obase, on);
            const int ge = min(a.out_grp[(size_t)me * (MAXD + 1) + d] - obase, on);
            for (int l = gs + sub; l < ge; l += NT) {
                const uint32_t c = a.out_code[obase + l];
                const bool bad = (int)(c >> 11) != d || (c & 0x7FFu) >= (uint32_t)H;
                if (bad) atomicAdd(a.err + 0, 1);
                ocode[l] = bad ? (uint16_t)0xFFFFu : (uint16_t)c;
                ow[l] = a.out_w[obase + l];
            }
        }
    }
    if (!first) {
        for (int k = tid; k < RING * HC * NS; k += nthr) part[k] = part_st[k];
        for (int k = tid; k < on; k += nthr) dw[k] = a.dwp[(size_t)q * a.nnz + obase + k];
        for (int k = tid; k < HC * R; k += nthr) dwo[k] = a.dwo_p[((size_t)q * H + h0) * R + k];
    }
    __shared__ int aborted;
    if (tid == 0) aborted = 0;
    __syncthreads();
    uint32_t *xcnt = a.xcnt + q;
    uint32_t target = 0;

    const size_t bq = (size_t)q * NS + SPT * sub;
    const bool ro = tid < NS * R;
    const int rb = ro ? tid / R : 0, rr = ro ? tid % R : 0;
    const float dmv = ro ? a.dm[(size_t)(q * NS + rb) * R + rr] : 0.f;
    const int tsv = ro ? a.tstar_in[(size_t)(q * NS + rb) * R + rr] : -1;
    float o = (ro && !first) ? a.o_st[(size_t)(q * NS + rb) * R + rr] : 0.f;
    float qp0 = 0.f, qp1 = 0.f;  // q[t + 1] of this thread's two samples
    if (nt && !first) {
        qp0 = a.q_st[bq * H + me];
        qp1 = a.q_st[(bq + 1) * H + me];
    }
    const int R4 = (R + NT - 1) / NT;

    // this neuron's 8 samples' spikes at step tt (0 before step 0): a byte of bits, or floats in the smooth model
    auto spikes_at = [&](int tt, float out[NS], uint32_t &byte) {
        byte = 0;
        if constexpr (SMOOTH) {
#pragma unroll
            for (int b = 0; b < NS; ++b) out[b] = 0.f;
            if (tt < 0 || !nt) return;
            const float4 *src = reinterpret_cast<const float4 *>(a.s_f) + (((size_t)tt * a.NC + q) * H + me) * 2;
            const float4 x = src[0], y = src[1];
            out[0] = x.x; out[1] = x.y; out[2] = x.z; out[3] = x.w;
            out[4] = y.x; out[5] = y.y; out[6] = y.z; out[7] = y.w;
            byte = 0xffu;
        } else {
            (void)out;
            if (tt < 0 || !nt) return;
            byte = a.s_bits[((size_t)tt * a.NC + q) * H + me];
        }
    };
    uint64_t hist = 0;      // spiking: byte d - 1 = the 8 samples' spikes at t - d
    float histf[MAXD][NS];  // smooth: histf[d - 1] = spikes at t - d
    for (int d = 1; d <= MAXD; ++d) {
        uint32_t byte;
        spikes_at(t1 - 1 - d, histf[d - 1], byte);
        if constexpr (!SMOOTH) hist |= (uint64_t)byte << (8 * (d - 1));
    }
    // the surrogate derivatives and spikes of the next step down, loaded one step ahead
    auto g_at = [&](int tt, int j) { return nt ? a.g_seg[((size_t)(tt - t0) * B + bq + j) * H + me] : 0.f; };
    float gn0 = g_at(t1 - 1, 0), gn1 = g_at(t1 - 1, 1);
    float stn[NS];
    uint32_t sbn;
    spikes_at(t1 - 1, stn, sbn);
    // outgoing rows of neuron me, delay group d, at step u (q[u] in pnew): partial[u - d] += w q[u][post];
    // dw += s[u - d][me] q[u][post] (sbyte, sf: the spikes at u - d). Every thread of the CTA calls it.
    auto out_rows = [&](int u, int d, uint32_t sbyte, const float *sf) {
        float acc[NS];
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[b] = 0.f;
        const int gs = nt ? grp[pl * (MAXD + 1) + d - 1] : 0, ge = nt ? grp[pl * (MAXD + 1) + d] : 0;
        if (__any_sync(FULL, sbyte != 0u))  // the same branch for the whole warp
            out_group<SMOOTH, true>(ocode, ow, pnew, dw, gs, ge, sub, sbyte != 0u, sbyte, sf, acc);
        else
            out_group<SMOOTH, false>(ocode, ow, pnew, dw, gs, ge, sub, false, 0u, sf, acc);
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[b] = __fadd_rn(acc[b], __shfl_xor_sync(FULL, acc[b], 1));
#pragma unroll
        for (int b = 0; b < NS; ++b) acc[b] = __fadd_rn(acc[b], __shfl_xor_sync(FULL, acc[b], 2));
        if (nt && u - d >= 0) {
            float x0, x1;
            mine(acc, sub, x0, x1);
            float *pp = part + ((size_t)((u - d) % RING) * HC + pl) * NS + SPT * sub;
            pp[0] = __fadd_rn(pp[0], x0);
            pp[1] = __fadd_rn(pp[1], x1);
        }
    };
    // the readout adjoint o[t] does not depend on q: it is made one step ahead, into the other half of obuf, so
    // that no barrier is needed for it (the half of o[t - 1] was last read at step t + 1, three barriers back)
    if (ro) {
        o = __fadd_rn(t1 - 1 == tsv ? dmv : 0.f, __fmul_rn(a.beta, o));
        obuf[(size_t)((t1 - 1) & 1) * NS * R + rb * R + rr] = o;
    }
    __syncthreads();  // o[t1 - 1] ready
    for (int t = t1 - 1; t >= t0; --t) {
        const float *ob = obuf + (size_t)(t & 1) * NS * R;  // o[t]
        float qv0 = 0.f, qv1 = 0.f;
        float st[NS];
#pragma unroll
        for (int b = 0; b < NS; ++b) st[b] = stn[b];
        const uint32_t sbyte_t = sbn;
        const float gc0 = gn0, gc1 = gn1;
        if (t > t0) {
            gn0 = g_at(t - 1, 0);
            gn1 = g_at(t - 1, 1);
            spikes_at(t - 1, stn, sbn);
        }
        if (nt) {
#pragma unroll
            for (int j = 0; j < SPT; ++j) {
                const int bl = SPT * sub + j;
                float *pp = part + ((size_t)(t % RING) * HC + pl) * NS + bl;
                float sh = *pp;
                for (int r = 0; r < R; ++r) sh = __fmaf_rn(__ldg(wout + pl * R + r), ob[bl * R + r], sh);
                *pp = 0.f;
                const float g = j ? gc1 : gc0;
                const float ap = __fmul_rn(a.alpha, j ? qp1 : qp0);
                const float qv = __fmaf_rn(g, __fmaf_rn(-a.theta, ap, sh), ap);
                a.dU[((size_t)t * B + bq + j) * H + me] = qv;
                if (j) qv1 = qv;
                else qv0 = qv;
            }
            qp0 = qv0;
            qp1 = qv1;
            // dw_out: this neuron's spikes at t times o[t]; each of its NT threads takes a quarter of the readouts
            if (sbyte_t) {
                for (int r = sub * R4; r < min(R, (sub + 1) * R4); ++r) {
                    float acc = dwo[pl * R + r];
                    for (int b = 0; b < NS; ++b) {
                        if constexpr (SMOOTH) acc = __fmaf_rn(st[b], ob[b * R + r], acc);
                        else if ((sbyte_t >> b) & 1u) acc = __fadd_rn(acc, ob[b * R + r]);
                    }
                    dwo[pl * R + r] = acc;
                }
            }
        }
        if (ro && t > t0) {  // o[t - 1]; o keeps o[t0] for the segment before this one
            o = __fadd_rn(t - 1 == tsv ? dmv : 0.f, __fmul_rn(a.beta, o));
            obuf[(size_t)((t - 1) & 1) * NS * R + rb * R + rr] = o;
        }
        float *slot = a.qx + ((size_t)q * 2 + (t & 1)) * H * NS;
        if (nt) reinterpret_cast<float2 *>(slot)[(size_t)me * (NS / 2) + sub] = make_float2(qv0, qv1);
        __syncthreads();  // this CTA's q[t] written
        target += CL;
        if (tid == 0) group_arrive(xcnt);
        // while the group's other CTAs arrive: step t + 1's delay groups 2..5 (pnew still holds q[t + 1]; their
        // partials are for steps t - 1 and earlier, so only the delay-1 group waits for q[t])
        if (t + 1 < t1) {
#pragma unroll
            for (int d = 2; d <= MAXD; ++d)
                out_rows(t + 1, d, SMOOTH ? 0xffu : (uint32_t)((hist >> (8 * (d - 2))) & 0xffu), histf[d - 2]);
        }
        if (tid == 0) group_wait(xcnt, target, a.err, a.wait_polls, aborted);
        __syncthreads();  // every CTA's q[t] written, every read of q[t + 1] done: copy q[t] (past L1) into pnew
        for (int j = tid; j < H * (NS / 4); j += nthr)
            reinterpret_cast<float4 *>(pnew)[(size_t)(j >> 1) * (QROW / 4) + (j & 1)] =
                __ldcg(reinterpret_cast<const float4 *>(slot) + j);
        __syncthreads();
        out_rows(t, 1, SMOOTH ? 0xffu : (uint32_t)(hist & 0xffu), histf[0]);
        // the spike history of step t - 1: delays 1..5 reach t - 2 .. t - 6
        if constexpr (SMOOTH) {
            for (int d = 1; d <= MAXD; ++d) {
                uint32_t byte;
                spikes_at(t - 1 - d, histf[d - 1], byte);
            }
        } else {
            uint32_t byte;
            spikes_at(t - 1 - MAXD, histf[0], byte);
            hist = (hist >> 8) | ((uint64_t)byte << (8 * (MAXD - 1)));
        }
    }
    // step t0's delay groups 2..5 (q[t0] is still in pnew)
#pragma unroll
    for (int d = 2; d <= MAXD; ++d)
        out_rows(t0, d, SMOOTH ? 0xffu : (uint32_t)((hist >> (8 * (d - 2))) & 0xffu), histf[d - 2]);
    // the state for the segment before this one
    __syncthreads();
    for (int k = tid; k < RING * HC * NS; k += nthr) part_st[k] = part[k];
    for (int k = tid; k < on; k += nthr) a.dwp[(size_t)q * a.nnz + obase + k] = dw[k];
    for (int k = tid; k < HC * R; k += nthr) a.dwo_p[((size_t)q * H + h0) * R + k] = dwo[k];
    if (nt) {
        a.q_st[bq * H + me] = qp0;
        a.q_st[(bq + 1) * H + me] = qp1;
    }
    if (ro && rank == 0) a.o_st[(size_t)(q * NS + rb) * R + rr] = o;
}

// dw_rec in the caller's (incoming, canonical) order: the clusters' partials added in cluster order.
__global__ void reduce_dw_kernel(const float *dwp, const int32_t *perm, int nnz, int NC, float *dw) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= nnz) return;
    float s = 0.f;
    for (int c = 0; c < NC; ++c) s = __fadd_rn(s, dwp[(size_t)c * nnz + l]);
    dw[perm[l]] = s;
}

__global__ void reduce_dwo_kernel(const float *dwo_p, int n, int NC, float *dwo) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float s = 0.f;
    for (int c = 0; c < NC; ++c) s = __fadd_rn(s, dwo_p[(size_t)c * n + k]);
    dwo[k] = s;
}

__global__ void gather_kernel(const float *src, const int32_t *perm, int n, float *dst) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l < n) dst[l] = src[perm[l]];
}

// ------------------------------------------------------------------------------------------------ input projection

// U[r] = sum over the spiking channels c of input row r (ascending) of w_in[c]: H / 4 threads per row, one float4
// of hidden units each, blockDim / (H / 4) rows per block; the channel indices of a row four at a time, then their
// weight rows. An index outside [0, C) adds nothing (the event lists are checked when they are built).
__global__ void __launch_bounds__(256) project_fwd_kernel(const int32_t *row_ptr, const int32_t *ch, int rows,
                                                          int C, int H, const float *w, float *u) {
    const int h4 = H / 4;
    const int r = blockIdx.x * (blockDim.x / h4) + threadIdx.x / h4, c4 = threadIdx.x % h4;
    if (r >= rows) return;
    const int k0 = row_ptr[r], k1 = row_ptr[r + 1];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int k = k0; k < k1; k += 4) {
        int c[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) c[j] = k + j < k1 ? __ldg(ch + k + j) : -1;
        float4 v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            v[j] = (c[j] >= 0 && c[j] < C) ? __ldg(reinterpret_cast<const float4 *>(w + (size_t)c[j] * H) + c4)
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (c[j] < 0 || c[j] >= C) continue;
            acc.x = __fadd_rn(acc.x, v[j].x);
            acc.y = __fadd_rn(acc.y, v[j].y);
            acc.z = __fadd_rn(acc.z, v[j].z);
            acc.w = __fadd_rn(acc.w, v[j].w);
        }
    }
    reinterpret_cast<float4 *>(u + (size_t)r * H)[c4] = acc;
}

// dw_in, first pass: chunk k (rows row_idx[chunk_ptr[k] .. chunk_ptr[k + 1]) of one channel, ascending) summed
// into partials[k]; a block per chunk, H / 4 threads, four rows' loads in flight. A row outside [0, rows) adds
// nothing.
__global__ void __launch_bounds__(256) project_bwd_chunk_kernel(const int32_t *chunk_ptr, const int32_t *row_idx,
                                                                int rows, int H, const float *du, float *partials) {
    const int k = blockIdx.x, c4 = threadIdx.x;
    const int j0 = chunk_ptr[k], j1 = chunk_ptr[k + 1];
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = j0; j < j1; j += 4) {
        int r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) r[i] = j + i < j1 ? __ldg(row_idx + j + i) : -1;
        float4 v[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
            v[i] = (r[i] >= 0 && r[i] < rows) ? __ldcs(reinterpret_cast<const float4 *>(du + (size_t)r[i] * H) + c4)
                                              : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (r[i] < 0 || r[i] >= rows) continue;
            acc.x = __fadd_rn(acc.x, v[i].x);
            acc.y = __fadd_rn(acc.y, v[i].y);
            acc.z = __fadd_rn(acc.z, v[i].z);
            acc.w = __fadd_rn(acc.w, v[i].w);
        }
    }
    reinterpret_cast<float4 *>(partials + (size_t)k * H)[c4] = acc;
}

// dw_in, second pass: channel c's chunks (ch_chunk[c] .. ch_chunk[c + 1]) added in chunk order.
__global__ void project_bwd_reduce_kernel(const int32_t *ch_chunk, int C, int H, const float *partials, float *dw) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)C * H) return;
    const int c = (int)(e / H), h = (int)(e % H);
    float s = 0.f;
    for (int k = ch_chunk[c]; k < ch_chunk[c + 1]; ++k) s = __fadd_rn(s, partials[(size_t)k * H + h]);
    dw[e] = s;
}

}  // namespace n2b_bptt

// ------------------------------------------------------------------------------------------------ host

namespace n2b_host {
int set_error(int code, const std::string &msg);
}

namespace {

using namespace n2b_bptt;

int bfail(int code, const std::string &msg) { return n2b_host::set_error(code, msg); }
int bcuda(cudaError_t e, const char *what) {
    return n2b_host::set_error(N2B_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define B_CUDA(call)                                    \
    do {                                                \
        cudaError_t _e = (call);                        \
        if (_e != cudaSuccess) return bcuda(_e, #call); \
    } while (0)

struct WsLayout {
    size_t spikes, vck, gseg, outw, dwp, dwo, part, qst, ost, qx, xcnt, err, total;
};

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

int check_desc(const n2b_bptt_desc *d) {
    if (!d) return bfail(N2B_EINVAL, "desc is NULL");
    if (d->batch <= 0 || d->batch % NS) return bfail(N2B_EINVAL, "batch must be a positive multiple of 8");
    if (d->hidden <= 0 || d->hidden % 32 || d->hidden > 1024)
        return bfail(N2B_EINVAL, "hidden must be a multiple of 32, at most 1024");
    if (d->readouts <= 0 || d->readouts > 32) return bfail(N2B_EINVAL, "readouts must be in 1..32");
    if (d->steps <= 0 || d->checkpoint <= 0) return bfail(N2B_EINVAL, "steps and checkpoint must be positive");
    if ((int64_t)d->steps * (d->batch / NS) * d->hidden >= ((int64_t)1 << 31))
        return bfail(N2B_EINVAL, "steps x batch / 8 x hidden must stay below 2^31");
    if (d->smooth && d->hidden > 256) return bfail(N2B_EINVAL, "the smooth model is for hidden <= 256");
    if (d->nnz < 0 || (d->nnz > 0 && (!d->in_code || !d->out_code || !d->out_perm)))
        return bfail(N2B_EINVAL, "missing link arrays");
    if (!d->in_ptr || !d->out_grp) return bfail(N2B_EINVAL, "missing row arrays");
    if (d->in_cta_max < 0 || d->out_cta_max < 0) return bfail(N2B_EINVAL, "negative link counts");
    if (d->wait_polls < 0) return bfail(N2B_EINVAL, "wait_polls < 0");
    return N2B_OK;
}

WsLayout ws_layout(const n2b_bptt_desc *d) {
    WsLayout L{};
    const size_t T = d->steps, B = d->batch, H = d->hidden, R = d->readouts, NC = B / NS;
    const size_t nseg = (T + d->checkpoint - 1) / d->checkpoint, K = std::min<size_t>(d->checkpoint, T);
    size_t o = 0;
    L.spikes = o; o = a256(o + (d->smooth ? sizeof(float) * T * NC * H * NS : T * NC * H));
    L.vck = o; o = a256(o + sizeof(float) * nseg * B * H);
    L.gseg = o; o = a256(o + sizeof(float) * 2 * K * B * H);  // two segments: one recomputed, one run back
    L.outw = o; o = a256(o + sizeof(float) * std::max<size_t>(d->nnz, 1));
    L.dwp = o; o = a256(o + sizeof(float) * NC * std::max<size_t>(d->nnz, 1));
    L.dwo = o; o = a256(o + sizeof(float) * NC * H * R);
    L.part = o; o = a256(o + sizeof(float) * NC * CL * RING * (H / CL) * NS);
    L.qst = o; o = a256(o + sizeof(float) * B * H);
    L.ost = o; o = a256(o + sizeof(float) * B * R);
    L.qx = o; o = a256(o + sizeof(float) * NC * 2 * H * NS);
    L.xcnt = o; o = a256(o + sizeof(uint32_t) * NC);
    L.err = o; o = a256(o + sizeof(int32_t) * N2B_BPTT_ERR_WORDS);
    L.total = o;
    return L;
}

int threads_of(const n2b_bptt_desc *d) {
    const int n = std::max(NT * (d->hidden / CL), NS * d->readouts);
    return (n + 31) / 32 * 32;
}

Args args_of(const n2b_bptt_desc *d, char *ws, const WsLayout &L) {
    Args a{};
    a.B = d->batch;
    a.T = d->steps;
    a.H = d->hidden;
    a.R = d->readouts;
    a.K = d->checkpoint;
    a.HC = d->hidden / CL;
    a.NC = d->batch / NS;
    a.nseg = (d->steps + d->checkpoint - 1) / d->checkpoint;
    a.nnz = d->nnz;
    a.alpha = d->alpha;
    a.beta = d->beta;
    a.theta = d->theta;
    a.slope = d->slope;
    a.in_ptr = d->in_ptr;
    a.in_code = d->in_code;
    a.out_grp = d->out_grp;
    a.out_code = d->out_code;
    a.s_bits = reinterpret_cast<uint8_t *>(ws + L.spikes);
    a.s_f = reinterpret_cast<float *>(ws + L.spikes);
    a.v_ckpt = reinterpret_cast<float *>(ws + L.vck);
    a.g_seg = reinterpret_cast<float *>(ws + L.gseg);
    a.out_w = reinterpret_cast<float *>(ws + L.outw);
    a.dwp = reinterpret_cast<float *>(ws + L.dwp);
    a.dwo_p = reinterpret_cast<float *>(ws + L.dwo);
    a.part_st = reinterpret_cast<float *>(ws + L.part);
    a.q_st = reinterpret_cast<float *>(ws + L.qst);
    a.o_st = reinterpret_cast<float *>(ws + L.ost);
    a.qx = reinterpret_cast<float *>(ws + L.qx);
    a.xcnt = reinterpret_cast<uint32_t *>(ws + L.xcnt);
    a.err = reinterpret_cast<int32_t *>(ws + L.err);
    a.wait_polls = d->wait_polls > 0 ? d->wait_polls : XCHG_SPIN_LIMIT;
    return a;
}

int check_ws(const n2b_bptt_desc *d, void *ws, size_t bytes, WsLayout &L) {
    int rc = check_desc(d);
    if (rc) return rc;
    L = ws_layout(d);
    if (!ws || (reinterpret_cast<uintptr_t>(ws) & 255)) return bfail(N2B_EINVAL, "workspace must be 256-byte aligned");
    if (bytes < L.total) return bfail(N2B_ESPACE, "workspace too small: need " + std::to_string(L.total) + " bytes");
    return N2B_OK;
}

template <class Kern, class... Rest>
int launch_cluster(Kern kern, int grid, int threads, size_t smem, cudaStream_t s, const Args &a, Rest... rest) {
    if (smem > 227 * 1024) return bfail(N2B_EINVAL, "shared memory need " + std::to_string(smem) + " bytes > 227 KiB");
    B_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    B_CUDA(cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
    if (clusters < 1) return bfail(N2B_ECUDA, "a cluster of 8 CTAs of this size cannot be resident");
    B_CUDA(cudaLaunchKernelEx(&cfg, kern, a, rest...));
    return N2B_OK;
}

// The groups of 8 CTAs that one cooperative launch of `kern` can hold (all resident at once).
template <class Kern>
int coop_groups(Kern kern, int threads, size_t smem, int &groups) {
    if (smem > 227 * 1024) return bfail(N2B_EINVAL, "shared memory need " + std::to_string(smem) + " bytes > 227 KiB");
    B_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 0, per_sm = 0;
    B_CUDA(cudaGetDevice(&dev));
    B_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem));
    groups = per_sm * sms / CL;
    if (groups < 1) return bfail(N2B_ECUDA, "a group of 8 CTAs of this size cannot be resident");
    return N2B_OK;
}

// The backward's two internal streams on a device, made on first use and kept: the adjoint on the highest
// priority, the next segment's recompute on the lowest, so that when both are ready the adjoint's CTAs are placed
// first and the recompute fills the SMs the adjoint leaves free.
struct SideStreams {
    cudaStream_t hi = nullptr, lo = nullptr;
};
int side_streams(SideStreams &out) {
    static std::mutex mu;
    static SideStreams per_dev[64];
    int dev = 0;
    B_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return bfail(N2B_EINVAL, "device index above 63");
    std::lock_guard<std::mutex> lock(mu);
    SideStreams &st = per_dev[dev];
    if (!st.hi) {
        int least = 0, greatest = 0;
        B_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        B_CUDA(cudaStreamCreateWithPriority(&st.hi, cudaStreamNonBlocking, greatest));
        B_CUDA(cudaStreamCreateWithPriority(&st.lo, cudaStreamNonBlocking, least));
    }
    out = st;
    return N2B_OK;
}

// Events of one backward call, destroyed on every return (pending work keeps them alive as long as it needs).
struct CallEvents {
    cudaEvent_t e[6] = {};
    ~CallEvents() {
        for (cudaEvent_t x : e)
            if (x) cudaEventDestroy(x);
    }
};

template <class Kern, class... Rest>
int launch_coop(Kern kern, int grid, int threads, size_t smem, cudaStream_t s, const Args &a, Rest... rest) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    B_CUDA(cudaLaunchKernelEx(&cfg, kern, a, rest...));
    return N2B_OK;
}

}  // namespace

extern "C" {

int n2b_bptt_workspace_bytes(const n2b_bptt_desc *d, size_t *bytes) {
    if (!bytes) return bfail(N2B_EINVAL, "bytes is NULL");
    int rc = check_desc(d);
    if (rc) return rc;
    *bytes = ws_layout(d).total;
    return N2B_OK;
}

int n2b_bptt_forward(const n2b_bptt_desc *d, const float *u, const float *w_rec, const float *w_out, int32_t tape,
                     float *m, int32_t *tstar, void *workspace, size_t workspace_bytes, void *stream) {
    WsLayout L;
    int rc = check_ws(d, workspace, workspace_bytes, L);
    if (rc) return rc;
    if (!u || !w_out || !m || !tstar || (d->nnz > 0 && !w_rec)) return bfail(N2B_EINVAL, "missing arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    Args a = args_of(d, ws, L);
    a.tape = tape != 0;
    a.U = u;
    a.in_w = w_rec;
    a.w_out = w_out;
    a.m = m;
    a.tstar = tstar;
    B_CUDA(cudaMemsetAsync(ws + L.err, 0, sizeof(int32_t) * N2B_BPTT_ERR_WORDS, s));
    const bool smooth = d->smooth != 0;
    FwdSmem S = fwd_smem(d->hidden, d->hidden / CL, d->readouts, smooth, true, d->in_cta_max);
    a.csr_smem = S.total <= 200 * 1024;
    if (!a.csr_smem) S = fwd_smem(d->hidden, d->hidden / CL, d->readouts, smooth, false, 0);
    const int grid = (d->batch / NS) * CL, threads = threads_of(d);
    return smooth ? launch_cluster(fwd_kernel<true>, grid, threads, S.total, s, a, d->in_cta_max)
                  : launch_cluster(fwd_kernel<false>, grid, threads, S.total, s, a, d->in_cta_max);
}

int n2b_bptt_backward(const n2b_bptt_desc *d, const float *u, const float *w_rec, const float *w_out,
                      const float *dm, const int32_t *tstar, float *du, float *dw_rec, float *dw_out,
                      void *workspace, size_t workspace_bytes, void *stream) {
    WsLayout L;
    int rc = check_ws(d, workspace, workspace_bytes, L);
    if (rc) return rc;
    if (!u || !w_out || !dm || !tstar || !du || !dw_out || (d->nnz > 0 && (!w_rec || !dw_rec)))
        return bfail(N2B_EINVAL, "missing arguments");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    Args a = args_of(d, ws, L);
    a.U = u;
    a.in_w = w_rec;
    a.w_out = w_out;
    a.dm = dm;
    a.tstar_in = tstar;
    a.dU = du;
    if (d->nnz > 0) {  // the weights in outgoing order
        gather_kernel<<<(d->nnz + 255) / 256, 256, 0, s>>>(w_rec, d->out_perm, d->nnz,
                                                           reinterpret_cast<float *>(ws + L.outw));
        B_CUDA(cudaGetLastError());
    }
    const bool smooth = d->smooth != 0;
    const BwdSmem S = bwd_smem(d->hidden, d->hidden / CL, d->readouts, d->out_cta_max);
    const int NC = d->batch / NS, threads = threads_of(d);
    const int K = d->checkpoint, nseg = a.nseg;
    const int rthreads = d->hidden % 64 == 0 ? 256 : 128;  // whole neurons of NT threads; hidden % 32 == 0
    const size_t rsmem = smooth ? 0 : (size_t)16 * d->hidden;  // the staged spike rows
    int per_launch = 0;  // groups per cooperative launch
    rc = smooth ? coop_groups(bwd_kernel<true>, threads, S.total, per_launch)
                : coop_groups(bwd_kernel<false>, threads, S.total, per_launch);
    if (rc) return rc;
    SideStreams st;
    rc = side_streams(st);
    if (rc) return rc;
    CallEvents ev;  // fork, recomputed[2], adjoint done[2], join
    for (cudaEvent_t &x : ev.e) B_CUDA(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    cudaEvent_t fork = ev.e[0], join = ev.e[5], *rec = ev.e + 1, *adj = ev.e + 3;
    B_CUDA(cudaEventRecord(fork, s));
    B_CUDA(cudaStreamWaitEvent(st.hi, fork, 0));
    B_CUDA(cudaStreamWaitEvent(st.lo, fork, 0));
    float *gbuf[2] = {a.g_seg, a.g_seg + (size_t)std::min(K, d->steps) * d->batch * d->hidden};
    // segment seg recomputed from its checkpoint into gbuf[seg & 1] on the low-priority stream
    auto recompute = [&](int seg) -> int {
        const int t0 = seg * K, t1 = std::min(d->steps, t0 + K);
        Args ra = a;
        ra.g_seg = gbuf[seg & 1];
        const dim3 rgrid((unsigned)(d->hidden / (rthreads / NT)), (unsigned)NC, (unsigned)((t1 - t0 + TC - 1) / TC));
        const unsigned vblocks = (unsigned)((d->batch * d->hidden + 255) / 256);
        if (smooth) {
            recompute_r_kernel<true><<<rgrid, rthreads, 0, st.lo>>>(ra, t0, t1);
            recompute_v_kernel<true><<<vblocks, 256, 0, st.lo>>>(ra, seg, t0, t1);
        } else {
            recompute_r_kernel<false><<<rgrid, rthreads, rsmem, st.lo>>>(ra, t0, t1);
            recompute_v_kernel<false><<<vblocks, 256, 0, st.lo>>>(ra, seg, t0, t1);
        }
        B_CUDA(cudaGetLastError());
        B_CUDA(cudaEventRecord(rec[seg & 1], st.lo));
        return N2B_OK;
    };
    // Segments run backwards. The recompute of segment seg - 1 overlaps the adjoint of seg; it reuses the buffer
    // of seg + 1, so it waits for that adjoint.
    rc = recompute(nseg - 1);
    if (rc) return rc;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int t0 = seg * K, t1 = std::min(d->steps, t0 + K);
        const int first = seg == nseg - 1;
        Args ba = a;
        ba.g_seg = gbuf[seg & 1];
        B_CUDA(cudaStreamWaitEvent(st.hi, rec[seg & 1], 0));
        B_CUDA(cudaMemsetAsync(a.xcnt, 0, sizeof(uint32_t) * NC, st.hi));
        for (int g0 = 0; g0 < NC; g0 += per_launch) {
            const int grid = std::min(per_launch, NC - g0) * CL;
            rc = smooth ? launch_coop(bwd_kernel<true>, grid, threads, S.total, st.hi, ba, d->out_cta_max, t0, t1,
                                      first, g0)
                        : launch_coop(bwd_kernel<false>, grid, threads, S.total, st.hi, ba, d->out_cta_max, t0, t1,
                                      first, g0);
            if (rc) return rc;
        }
        B_CUDA(cudaEventRecord(adj[seg & 1], st.hi));
        if (seg > 0) {
            if (seg + 1 < nseg) B_CUDA(cudaStreamWaitEvent(st.lo, adj[(seg + 1) & 1], 0));
            rc = recompute(seg - 1);
            if (rc) return rc;
        }
    }
    if (d->nnz > 0) {
        reduce_dw_kernel<<<(d->nnz + 255) / 256, 256, 0, st.hi>>>(a.dwp, d->out_perm, d->nnz, NC, dw_rec);
        B_CUDA(cudaGetLastError());
    }
    const int n = d->hidden * d->readouts;
    reduce_dwo_kernel<<<(n + 255) / 256, 256, 0, st.hi>>>(a.dwo_p, n, NC, dw_out);
    B_CUDA(cudaGetLastError());
    B_CUDA(cudaEventRecord(join, st.hi));
    B_CUDA(cudaStreamWaitEvent(s, join, 0));
    return N2B_OK;
}

int n2b_bptt_status(const n2b_bptt_desc *d, void *workspace, size_t workspace_bytes, int32_t *words, void *stream) {
    WsLayout L;
    int rc = check_ws(d, workspace, workspace_bytes, L);
    if (rc) return rc;
    if (!words) return bfail(N2B_EINVAL, "words is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int32_t host[N2B_BPTT_ERR_WORDS];
    B_CUDA(cudaMemcpyAsync(host, static_cast<char *>(workspace) + L.err, sizeof(host), cudaMemcpyDeviceToHost, s));
    B_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < N2B_BPTT_ERR_WORDS; ++k) words[k] = host[k];
    return N2B_OK;
}

int n2b_bptt_spikes(const n2b_bptt_desc *d, void *workspace, size_t workspace_bytes, void *out, void *stream) {
    WsLayout L;
    int rc = check_ws(d, workspace, workspace_bytes, L);
    if (rc) return rc;
    if (!out) return bfail(N2B_EINVAL, "out is NULL");
    const size_t T = d->steps, NC = d->batch / NS, H = d->hidden;
    const size_t n = d->smooth ? sizeof(float) * T * NC * H * NS : T * NC * H;
    B_CUDA(cudaMemcpyAsync(out, static_cast<char *>(workspace) + L.spikes, n, cudaMemcpyDeviceToDevice,
                           reinterpret_cast<cudaStream_t>(stream)));
    return N2B_OK;
}

int n2b_project_forward(const int32_t *row_ptr, const int32_t *channel, int32_t rows, int32_t channels,
                        int32_t hidden, const float *w_in, float *u, void *stream) {
    if (rows < 0 || channels <= 0 || hidden <= 0 || hidden % 4 || hidden > 1024)
        return bfail(N2B_EINVAL, "project: rows >= 0, channels > 0, hidden a multiple of 4 up to 1024");
    if (rows == 0) return N2B_OK;
    if (!row_ptr || !channel || !w_in || !u) return bfail(N2B_EINVAL, "project: missing arguments");
    if ((reinterpret_cast<uintptr_t>(w_in) | reinterpret_cast<uintptr_t>(u)) & 15)
        return bfail(N2B_EINVAL, "project: w_in and u must be 16-byte aligned");
    const int h4 = hidden / 4, rpb = std::max(1, 256 / h4);
    project_fwd_kernel<<<(unsigned)((rows + rpb - 1) / rpb), (unsigned)(rpb * h4), 0,
                         reinterpret_cast<cudaStream_t>(stream)>>>(row_ptr, channel, rows, channels, hidden, w_in, u);
    B_CUDA(cudaGetLastError());
    return N2B_OK;
}

int n2b_project_backward(const int32_t *chunk_ptr, int32_t n_chunks, const int32_t *row_idx,
                         const int32_t *channel_chunk, int32_t channels, int32_t rows, int32_t hidden,
                         const float *du, float *partials, float *dw_in, void *stream) {
    if (n_chunks < 0 || rows < 0 || channels <= 0 || hidden <= 0 || hidden % 4 || hidden > 1024)
        return bfail(N2B_EINVAL, "project: n_chunks, rows >= 0, channels > 0, hidden a multiple of 4 up to 1024");
    if (!channel_chunk || !dw_in || (n_chunks > 0 && (!chunk_ptr || !row_idx || !du || !partials)))
        return bfail(N2B_EINVAL, "project: missing arguments");
    if ((reinterpret_cast<uintptr_t>(du) | reinterpret_cast<uintptr_t>(partials)) & 15)
        return bfail(N2B_EINVAL, "project: du and partials must be 16-byte aligned");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n_chunks > 0) {
        project_bwd_chunk_kernel<<<(unsigned)n_chunks, (unsigned)(hidden / 4), 0, s>>>(chunk_ptr, row_idx, rows,
                                                                                     hidden, du, partials);
        B_CUDA(cudaGetLastError());
    }
    const size_t n = (size_t)channels * hidden;
    project_bwd_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(channel_chunk, channels, hidden, partials,
                                                                          dw_in);
    B_CUDA(cudaGetLastError());
    return N2B_OK;
}

}  // extern "C"
