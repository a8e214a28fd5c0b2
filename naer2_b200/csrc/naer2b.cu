// naer2b: the C ABI of the fixed-dt hot path (include/naer2b.h).
//
// Host side: validates the caller's description, lays the device tables out
// in the caller's workspace (PopDev per population, ConnDev per connection
// grouped by source for push and by target for pull, one tile per block),
// launches the step kernel once per step (plus one counter advance per
// call), and captures windows of steps into CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/naer2b.h"
#include "n2b_device.cuh"

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
    g_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(N2B_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define N2B_CUDA(call)                                      \
    do {                                                    \
        cudaError_t _e = (call);                            \
        if (_e != cudaSuccess) return cuda_fail(_e, #call); \
    } while (0)

bool pow2(int32_t x) { return x > 0 && (x & (x - 1)) == 0; }

// The calling thread's current device, put back when an entry point returns (each one makes its handle's
// device current for its work).
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

// The calling thread's error message, shared with the library's other translation units (bptt.cu).
namespace n2b_host {
int set_error(int code, const std::string &msg) { return fail(code, msg); }
}  // namespace n2b_host

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
    size_t pops, push, pull, tiles, step, rec0, err, counters, items, item_count, barrier, pull_rows, total;
    int32_t n_push, n_pull, n_tiles, item_cap;
};

int32_t block_of(const n2b_options *opt) {
    int32_t b = opt && opt->block ? opt->block : 128;
    return b;
}

Layout layout(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
              int32_t block) {
    Layout L{};
    // work items of one step at most: every row's deferred links in items of `block` links, every source firing
    int64_t cap = 1;
    for (int32_t c = 0; c < n_conns; ++c) {
        (conns[c].mode == N2B_PULL ? L.n_pull : L.n_push) += 1;
        if (conns[c].mode == N2B_PUSH && conns[c].split)
            cap += (int64_t)conns[c].n_links / block + pops[conns[c].src].n + 1;
    }
    L.item_cap = (int32_t)std::min<int64_t>(cap, (int64_t)1 << 30);
    int64_t item_rows = 0;  // the grid-wide pull's items' first rows: PULL_ITEM links each, at most
    for (int32_t c = 0; c < n_conns; ++c)
        if (conns[c].mode == N2B_PULL && conns[c].split) item_rows += conns[c].n_links / n2b::PULL_ITEM + 2;
    for (int32_t p = 0; p < n_pops; ++p) L.n_tiles += (pops[p].n + block - 1) / block;
    size_t o = 0;
    L.pops = o; o = align256(o + sizeof(n2b::PopDev) * std::max(n_pops, 1));
    L.push = o; o = align256(o + sizeof(n2b::ConnDev) * std::max(L.n_push, 1));
    L.pull = o; o = align256(o + sizeof(n2b::ConnDev) * std::max(L.n_pull, 1));
    L.tiles = o; o = align256(o + sizeof(int4) * std::max(L.n_tiles, 1));
    L.step = o; o = align256(o + sizeof(long long));
    L.rec0 = o; o = align256(o + sizeof(long long));
    L.err = o; o = align256(o + sizeof(int32_t) * N2B_ERR_WORDS);
    L.counters = o; o = align256(o + sizeof(unsigned long long) * (2 + std::max(n_pops, 1)));
    L.item_count = o; o = align256(o + sizeof(int32_t) * 12);  // list lengths, tile, far-chunk, pull counters
    L.items = o; o = align256(o + sizeof(int4) * 3 * (size_t)L.item_cap);
    L.barrier = o; o = align256(o + sizeof(unsigned) * n2b::BAR_WORDS);
    L.pull_rows = o; o = align256(o + sizeof(int32_t) * (size_t)std::max<int64_t>(item_rows, 1));
    L.total = o;
    return L;
}

int validate(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
             const n2b_options *opt) {
    if (n_pops < 0 || n_conns < 0 || (n_pops > 0 && !pops) || (n_conns > 0 && !conns))
        return fail(N2B_EINVAL, "negative counts or missing arrays");
    const int32_t block = block_of(opt);
    if (block != 64 && block != 128 && block != 256) return fail(N2B_EINVAL, "block must be 64, 128 or 256");
    if (opt && opt->barrier_limit_ns < 0) return fail(N2B_EINVAL, "barrier_limit_ns < 0");
    for (int32_t p = 0; p < n_pops; ++p) {
        const n2b_population &P = pops[p];
        const std::string at = "population " + std::to_string(p) + ": ";
        if (P.n < 0 || P.n > (1 << 24)) return fail(N2B_EINVAL, at + "n must be in [0, 2^24]");
        if (P.model != N2B_MODEL_LIF_DELTA && P.model != N2B_MODEL_PD14 && P.model != N2B_MODEL_POISSON_SOURCE)
            return fail(N2B_EINVAL, at + "unknown model");
        if (P.shift < 0 || P.shift > 62) return fail(N2B_EINVAL, at + "shift must be in [0, 62]");
        if (P.bit_depth != 0 && (!pow2(P.bit_depth) || P.bit_depth > 256 || !P.bits))
            return fail(N2B_EINVAL, at + "bit_depth must be 0 or a power of two <= 256 with bits");
        if (P.raster_steps < 0 || (P.raster_steps > 0 && !P.raster))
            return fail(N2B_EINVAL, at + "raster_steps > 0 needs a raster");
        if (P.n == 0) continue;
        if (P.model != N2B_MODEL_POISSON_SOURCE) {
            if (!pow2(P.acc_depth) || P.acc_depth > 256 || !P.acc)
                return fail(N2B_EINVAL, at + "acc_depth must be a power of two <= 256 with acc");
            if (!P.v || !P.ref || (P.model == N2B_MODEL_PD14 && !P.i))
                return fail(N2B_EINVAL, at + "missing state arrays");
            if (P.ext_len < 0 || (P.ext_len > 0 && !P.ext_table))
                return fail(N2B_EINVAL, at + "ext_len > 0 needs ext_table");
        }
    }
    for (int32_t c = 0; c < n_conns; ++c) {
        const n2b_connection &C = conns[c];
        const std::string at = "connection " + std::to_string(c) + ": ";
        if (C.src < 0 || C.src >= n_pops || C.tgt < 0 || C.tgt >= n_pops)
            return fail(N2B_EINVAL, at + "src/tgt out of range");
        if (C.mode != N2B_PUSH && C.mode != N2B_PULL) return fail(N2B_EINVAL, at + "unknown mode");
        if (C.n_links < 0 || !C.ptr || (C.n_links > 0 && !C.link))
            return fail(N2B_EINVAL, at + "missing CSR arrays");
        const n2b_population &T = pops[C.tgt];
        const n2b_population &S = pops[C.src];
        if (T.model == N2B_MODEL_POISSON_SOURCE) return fail(N2B_EINVAL, at + "a Poisson source takes no input");
        if (T.n > 0 && (!T.acc || !pow2(T.acc_depth))) return fail(N2B_EINVAL, at + "target has no arrival slots");
        if (C.mode == N2B_PULL && S.n > 0 && (!S.bits || !pow2(S.bit_depth)))
            return fail(N2B_EINVAL, at + "a pull connection needs the source's spike-bit ring");
        if (S.n > 0 && (int64_t)C.n_links > ((int64_t)1 << 31) - 1) return fail(N2B_EINVAL, at + "more than 2^31 links");
    }
    return N2B_OK;
}

}  // namespace

struct n2b_net {
    int device = 0;
    int32_t block = 128;
    int32_t grid = 0;
    int32_t persistent = 0;
    int32_t inl = 0;  // tables in the kernel parameters
    int32_t dense = 0;  // persistent windows: the three-blocks-per-SM kernel (more tiles than two per SM hold)
    int32_t n_pops = 0;
    size_t dyn_smem = 0;  // dynamic shared memory of the step kernels (the staged pull's buffers)
    Layout L{};
    char *ws = nullptr;
    n2b::StepArgs args{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int32_t window = 0;
};

namespace {

template <int NPB, bool INL>
cudaError_t launch_one(n2b_net *net, int64_t n_steps, cudaStream_t s) {
    if (net->persistent) {
        int32_t k = (int32_t)n_steps;
        void *args[] = {(void *)&net->args, (void *)&k};
        const void *kern = net->dense ? (const void *)n2b::persistent_kernel<NPB, INL, true>
                                      : (const void *)n2b::persistent_kernel<NPB, INL, false>;
        return cudaLaunchCooperativeKernel(kern, dim3(net->grid), dim3(NPB), args, net->dyn_smem, s);
    }
    n2b::StepArgs &a = net->args;
    for (int64_t k = 0; k < n_steps; ++k) {
        a.offset = (int32_t)k;
        n2b::step_kernel<NPB, INL><<<net->grid, NPB, net->dyn_smem, s>>>(a);
    }
    a.offset = 0;
    return cudaGetLastError();
}

template <bool INL>
cudaError_t launch_block(n2b_net *net, int64_t n_steps, cudaStream_t s) {
    switch (net->block) {
        case 64: return launch_one<64, INL>(net, n_steps, s);
        case 256: return launch_one<256, INL>(net, n_steps, s);
        default: return launch_one<128, INL>(net, n_steps, s);
    }
}

cudaError_t launch_steps(n2b_net *net, int64_t n_steps, cudaStream_t s) {
    if (net->L.n_tiles > 0 && n_steps > 0) {
        cudaError_t e = net->inl ? launch_block<true>(net, n_steps, s) : launch_block<false>(net, n_steps, s);
        if (e != cudaSuccess) return e;
    }
    n2b::advance_kernel<<<1, 1, 0, s>>>(reinterpret_cast<long long *>(net->ws + net->L.step), n_steps,
                                        reinterpret_cast<unsigned *>(net->ws + net->L.barrier));
    return cudaGetLastError();
}

// The step kernels' dynamic shared memory limit raised to `dyn` (the staged pull's buffers), and the persistent
// kernel's resident blocks per SM with it.
template <int NPB, bool INL, bool DENSE>
cudaError_t occupancy(int *per_sm, size_t dyn) {
    const void *pk = (const void *)n2b::persistent_kernel<NPB, INL, DENSE>;
    cudaError_t e = cudaFuncSetAttribute(pk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute((const void *)n2b::step_kernel<NPB, INL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)dyn);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, pk, NPB, dyn);
}

template <bool DENSE>
cudaError_t occupancy_of(int32_t block, bool inl, size_t dyn, int *per_sm) {
    switch (block) {
        case 64: return inl ? occupancy<64, true, DENSE>(per_sm, dyn) : occupancy<64, false, DENSE>(per_sm, dyn);
        case 256: return inl ? occupancy<256, true, DENSE>(per_sm, dyn) : occupancy<256, false, DENSE>(per_sm, dyn);
        default: return inl ? occupancy<128, true, DENSE>(per_sm, dyn) : occupancy<128, false, DENSE>(per_sm, dyn);
    }
}

int coresident_blocks(int32_t block, bool inl, bool dense, int device, size_t dyn, int *out) {
    int per_sm = 0, sms = 0;
    cudaError_t e = dense ? occupancy_of<true>(block, inl, dyn, &per_sm) : occupancy_of<false>(block, inl, dyn, &per_sm);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    *out = per_sm * sms;
    return N2B_OK;
}

void drop_graph(n2b_net *net) {
    if (net->exec) cudaGraphExecDestroy(net->exec);
    if (net->graph) cudaGraphDestroy(net->graph);
    net->exec = nullptr;
    net->graph = nullptr;
    net->window = 0;
}

}  // namespace

extern "C" {

int32_t n2b_abi_version(void) { return N2B_ABI_VERSION; }

const char *n2b_last_error(void) { return g_error.c_str(); }

int n2b_workspace_bytes(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
                        const n2b_options *opt, size_t *bytes) {
    if (!bytes) return fail(N2B_EINVAL, "bytes is NULL");
    int rc = validate(pops, n_pops, conns, n_conns, opt);
    if (rc) return rc;
    *bytes = layout(pops, n_pops, conns, n_conns, block_of(opt)).total;
    return N2B_OK;
}

int n2b_create(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns, int32_t n_conns,
               const n2b_options *opt, void *workspace, size_t workspace_bytes, void *stream, n2b_net **out) {
    DeviceGuard guard;
    if (!out) return fail(N2B_EINVAL, "out is NULL");
    *out = nullptr;
    int rc = validate(pops, n_pops, conns, n_conns, opt);
    if (rc) return rc;
    const int32_t block = block_of(opt);
    Layout L = layout(pops, n_pops, conns, n_conns, block);
    if (!workspace || (reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return fail(N2B_EINVAL, "workspace must be a 256-byte aligned device pointer");
    if (workspace_bytes < L.total)
        return fail(N2B_ESPACE, "workspace too small: need " + std::to_string(L.total) + " bytes");
    const int device = opt ? opt->device : 0;
    N2B_CUDA(cudaSetDevice(device));

    // host images of the tables
    std::vector<n2b::PopDev> pd(std::max(n_pops, 1));
    std::vector<n2b::ConnDev> push, pull;
    std::vector<int4> tiles;
    for (int32_t p = 0; p < n_pops; ++p) {
        const n2b_population &P = pops[p];
        n2b::PopDev &D = pd[p];
        std::memset(&D, 0, sizeof(D));
        D.model = P.model;
        D.n = P.n;
        D.acc_mask = P.acc_depth > 0 ? P.acc_depth - 1 : 0;
        D.bit_mask = P.bit_depth > 0 ? P.bit_depth - 1 : 0;
        D.words = (P.n + 31) / 32;
        D.shift = P.shift;
        D.ref_steps = P.ref_steps;
        D.ext_len = P.ext_len;
        D.fire_threshold = P.fire_threshold;
        D.seed_lo = (uint32_t)P.seed;
        D.seed_hi = (uint32_t)(P.seed >> 32);
        D.index = (uint32_t)p;
        D.ext_wfx = P.ext_wfx;
        D.inv_scale = std::ldexp(1.0f, -P.shift);
        for (int k = 0; k < 8; ++k) D.p[k] = P.p[k];
        D.v = P.v;
        D.i = P.i;
        D.ref = P.ref;
        D.acc = reinterpret_cast<long long *>(P.acc);
        D.bits = P.bits;
        D.ext_table = P.ext_table;
        D.raster = P.raster;
        D.raster_steps = P.raster_steps;
    }
    auto conn_dev = [&](const n2b_connection &C) {
        n2b::ConnDev D;
        std::memset(&D, 0, sizeof(D));
        const n2b_population &S = pops[C.src], &T = pops[C.tgt];
        D.homogeneous = C.w == nullptr;
        D.src_n = S.n;
        D.tgt_n = T.n;
        D.tgt_acc_mask = T.acc_depth > 0 ? T.acc_depth - 1 : 0;
        D.src_bit_mask = S.bit_depth > 0 ? S.bit_depth - 1 : 0;
        D.src_words = (S.n + 31) / 32;
        D.wscale = std::ldexp(1.0f, T.shift);
        D.wfx = (long long)std::nearbyint((double)std::ldexp(C.weight, T.shift));
        D.ptr = C.ptr;
        D.link = C.link;
        D.w = C.w;
        D.tgt_acc = reinterpret_cast<long long *>(T.acc);
        D.src_bits = S.bits;
        D.has_split = C.split != nullptr;
        D.split = C.split;
        D.ring_off = -1;
        D.n_links = C.n_links;
        // pull rows stream through shared memory by bulk copies, which need 16-byte aligned sources
        D.staged = C.mode == N2B_PULL && (reinterpret_cast<uintptr_t>(C.link) & 15) == 0 &&
                   (C.w == nullptr || (reinterpret_cast<uintptr_t>(C.w) & 15) == 0);
        return D;
    };
    for (int32_t p = 0; p < n_pops; ++p) {
        pd[p].out_first = (int32_t)push.size();
        for (int32_t c = 0; c < n_conns; ++c)
            if (conns[c].mode == N2B_PUSH && conns[c].src == p) push.push_back(conn_dev(conns[c]));
        pd[p].n_out = (int32_t)push.size() - pd[p].out_first;
        pd[p].pull_first = (int32_t)pull.size();
        for (int32_t c = 0; c < n_conns; ++c)
            if (conns[c].mode == N2B_PULL && conns[c].tgt == p) pull.push_back(conn_dev(conns[c]));
        pd[p].n_pull = (int32_t)pull.size() - pd[p].pull_first;
    }
    // the pull: a PullStage per warp in dynamic shared memory when the network has pull connections, and after
    // them a ring cache -- for the largest pull source's spike-bit ring (the in-step pull, one connection at a
    // time) and, when they fit together, every split connection's source ring at its ring_off (the grid-wide
    // pull), up to RING_CACHE_MAX words; the grid-wide pull's items, PULL_ITEM links each, numbered by
    // connection, their first rows found by a set-up kernel
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    // a split pull connection's first delay >= 2 link (read back once) and its items of PULL_ITEM links
    std::vector<int32_t> far0(pull.size(), 0);
    for (size_t c = 0; c < pull.size(); ++c)
        if (pull[c].has_split && pull[c].tgt_n > 0)
            N2B_CUDA(cudaMemcpyAsync(&far0[c], pull[c].split, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    N2B_CUDA(cudaStreamSynchronize(s));
    int32_t max_ring = 0, total_ring = 0, pull_items = 0;
    size_t item_rows = 0;
    for (size_t c = 0; c < pull.size(); ++c) {
        n2b::ConnDev &C = pull[c];
        const int32_t w = (C.src_bit_mask + 1) * C.src_words;
        max_ring = std::max(max_ring, w);
        if (C.has_split) {
            if (far0[c] < 0 || far0[c] > C.n_links)
                return fail(N2B_EINVAL, "a pull connection's split offsets lie outside its links");
            for (size_t e = 0; e < c && C.ring_off < 0; ++e)  // a source ring already in the cache is shared
                if (pull[e].has_split && pull[e].src_bits == C.src_bits) C.ring_off = pull[e].ring_off;
            if (C.ring_off < 0) {
                C.ring_off = total_ring;
                total_ring += w;
            }
            C.far0 = far0[c];
            C.item0 = pull_items;
            C.n_items = (C.tgt_n > 0 && far0[c] < C.n_links)
                            ? (C.n_links + n2b::PULL_ITEM - 1) / n2b::PULL_ITEM - far0[c] / n2b::PULL_ITEM
                            : 0;
            C.item_row = reinterpret_cast<const int32_t *>(ws + L.pull_rows) + item_rows;
            item_rows += (size_t)C.n_items;
            pull_items += C.n_items;
        }
    }
    const int32_t ring_words = max_ring <= n2b::RING_CACHE_MAX ? max_ring : 0;  // 0: sources read from global
    const bool ring_all = total_ring > 0 && total_ring <= n2b::RING_CACHE_MAX;
    if (!ring_all)
        for (n2b::ConnDev &C : pull) C.ring_off = -1;
    const int32_t cache_words = std::max(ring_words, ring_all ? total_ring : 0);
    // tiles: the largest populations' first (their blocks start first)
    std::vector<int32_t> order(n_pops);
    for (int32_t p = 0; p < n_pops; ++p) order[p] = p;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return pops[x].n > pops[y].n; });
    for (int32_t p : order)
        for (int32_t f = 0; f < pops[p].n; f += block) tiles.push_back(make_int4(p, f, std::min(block, pops[p].n - f), 0));

    // the first entries of every Poisson table, inline (read back once)
    for (int32_t p = 0; p < n_pops; ++p) {
        const int32_t k = std::min(pops[p].ext_len, n2b::EXT_INLINE);
        if (pops[p].n > 0 && k > 0)
            N2B_CUDA(cudaMemcpyAsync(pd[p].ext_tab, pops[p].ext_table, sizeof(uint32_t) * k, cudaMemcpyDeviceToHost, s));
    }
    N2B_CUDA(cudaStreamSynchronize(s));
    if (n_pops) N2B_CUDA(cudaMemcpyAsync(ws + L.pops, pd.data(), sizeof(n2b::PopDev) * n_pops, cudaMemcpyHostToDevice, s));
    if (!push.empty())
        N2B_CUDA(cudaMemcpyAsync(ws + L.push, push.data(), sizeof(n2b::ConnDev) * push.size(), cudaMemcpyHostToDevice, s));
    if (!pull.empty())
        N2B_CUDA(cudaMemcpyAsync(ws + L.pull, pull.data(), sizeof(n2b::ConnDev) * pull.size(), cudaMemcpyHostToDevice, s));
    if (!tiles.empty())
        N2B_CUDA(cudaMemcpyAsync(ws + L.tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice, s));
    for (const n2b::ConnDev &C : pull)
        if (C.n_items > 0)
            n2b::pull_item_rows_kernel<<<(C.n_items + 127) / 128, 128, 0, s>>>(
                C.split, C.tgt_n, C.far0, C.n_items, const_cast<int32_t *>(C.item_row));
    n2b::set_step_kernel<<<1, 1, 0, s>>>(reinterpret_cast<long long *>(ws + L.step), 0,
                                         reinterpret_cast<int32_t *>(ws + L.item_count));
    n2b::set_kernel<<<1, 1, 0, s>>>(reinterpret_cast<long long *>(ws + L.rec0), 0);
    n2b::zero_kernel<<<1, 64, 0, s>>>(reinterpret_cast<int32_t *>(ws + L.err), N2B_ERR_WORDS,
                                      reinterpret_cast<unsigned long long *>(ws + L.counters), 2 + n_pops);
    N2B_CUDA(cudaMemsetAsync(ws + L.barrier, 0, sizeof(unsigned) * n2b::BAR_WORDS, s));
    N2B_CUDA(cudaGetLastError());
    // the host images are read by the copies above: wait for them before they go
    N2B_CUDA(cudaStreamSynchronize(s));

    int sms = 0;
    N2B_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int persistent = opt && opt->persistent;
    const bool inl = n_pops <= n2b::INLINE_POPS && (int32_t)push.size() <= n2b::INLINE_PUSH &&
                     (int32_t)pull.size() <= n2b::INLINE_PULL;
    // default: per-step launches two blocks per SM; persistent windows one per SM, and at least one per tile
    // plus half an SM's worth of tile-free blocks for the far links (capped by what can be resident; a
    // smaller grid makes the grid barrier cheaper: config 1 steps 2-4% faster at 148 blocks than at 296)
    int want = (opt && opt->grid > 0) ? opt->grid
                                      : (persistent ? std::max(sms, L.n_tiles + sms / 2) : 2 * sms);
    int grid = std::max(L.n_tiles, want);
    bool weighted_pull = false;
    for (const n2b::ConnDev &C : pull) weighted_pull = weighted_pull || !C.homogeneous;
    const size_t stage_bytes = n2b::pull_stage_bytes(weighted_pull);
    const size_t dyn = pull.empty() ? 0 : stage_bytes * (size_t)(block / 32) + sizeof(uint32_t) * cache_words;
    int most = 0;
    int rc2 = coresident_blocks(block, inl, false, device, dyn, &most);  // also raises the kernels' dynamic limit
    if (rc2) return rc2;
    bool dense = false;
    if (persistent && L.n_tiles > most && pull.empty()) {  // more tiles than blocks: the denser kernel (push only)
        int most3 = 0;
        rc2 = coresident_blocks(block, inl, true, device, dyn, &most3);
        if (rc2) return rc2;
        if (most3 > most) {
            dense = true;
            most = most3;
        }
    }
    if (persistent) {
        if (most < 1) return fail(N2B_ECUDA, "the persistent kernel cannot be resident");
        // a grid-wide pull is spread over every warp of the launch, and the dense kernel's tile-free blocks take
        // the far items (PD14: 7.17 us per step at 444 blocks against 7.65 at 379): by default as many blocks
        // as can be resident
        if ((pull_items > 0 || dense) && !(opt && opt->grid > 0)) want = most;
        grid = std::min(std::min(want, most), n2b::BAR_MAX_BLOCKS);
        grid = std::max(grid, 1);
    }
    n2b_net *net = new n2b_net();
    net->device = device;
    net->block = block;
    net->persistent = persistent;
    net->inl = inl;
    net->grid = grid;
    net->n_pops = n_pops;
    net->dyn_smem = dyn;
    net->dense = dense;
    net->L = L;
    net->ws = ws;
    n2b::StepArgs &a = net->args;
    a.pops = reinterpret_cast<const n2b::PopDev *>(ws + L.pops);
    a.push = reinterpret_cast<const n2b::ConnDev *>(ws + L.push);
    a.pull = reinterpret_cast<const n2b::ConnDev *>(ws + L.pull);
    a.tiles = reinterpret_cast<const int4 *>(ws + L.tiles);
    a.step = reinterpret_cast<const long long *>(ws + L.step);
    a.rec0 = reinterpret_cast<const long long *>(ws + L.rec0);
    a.err = reinterpret_cast<int32_t *>(ws + L.err);
    a.counters = reinterpret_cast<unsigned long long *>(ws + L.counters);
    a.items = reinterpret_cast<int4 *>(ws + L.items);
    a.item_count = reinterpret_cast<int32_t *>(ws + L.item_count);
    a.tile_claim = a.item_count + 3;
    a.pull_claim = a.item_count + 9;
    a.item_cap = L.item_cap;
    a.n_tiles = L.n_tiles;
    a.offset = 0;
    a.barrier = reinterpret_cast<unsigned *>(ws + L.barrier);
    a.bar_limit_ns = (opt && opt->barrier_limit_ns > 0) ? (unsigned long long)opt->barrier_limit_ns
                                                         : n2b::BAR_LIMIT_NS;
    a.pull_staged = dyn > 0;
    a.pull_stage_bytes = (int32_t)stage_bytes;
    a.ring_cache_words = ring_words;
    a.ring_cache_all = ring_all;
    a.pull_items = pull_items;
    a.n_pull = (int32_t)pull.size();
    a.n_pops = n_pops;
    a.n_push = L.n_push;
    if (inl) {
        // inline: tiles in population order (the global table lists the largest populations first)
        int32_t t = 0;
        for (int32_t p = 0; p < n_pops; ++p) {
            a.tile_first[p] = t;
            t += (pops[p].n + block - 1) / block;
            a.pops_i[p] = pd[p];
        }
        a.tile_first[n_pops] = t;
        for (size_t c = 0; c < push.size(); ++c) a.push_i[c] = push[c];
        for (size_t c = 0; c < pull.size(); ++c) a.pull_i[c] = pull[c];
    }
    *out = net;
    return N2B_OK;
}

int n2b_step(n2b_net *net, int64_t n_steps, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    if (n_steps < 0 || n_steps > (int64_t)1 << 30) return fail(N2B_EINVAL, "n_steps out of range");
    N2B_CUDA(cudaSetDevice(net->device));
    cudaError_t e = launch_steps(net, n_steps, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_fail(e, "step launch");
    return N2B_OK;
}

int n2b_capture(n2b_net *net, int32_t window_steps, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    if (window_steps <= 0 || window_steps > (1 << 20)) return fail(N2B_EINVAL, "window_steps out of range");
    N2B_CUDA(cudaSetDevice(net->device));
    drop_graph(net);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    N2B_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = launch_steps(net, window_steps, s);
    cudaGraph_t g = nullptr;
    cudaError_t ee = cudaStreamEndCapture(s, &g);
    if (le != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return cuda_fail(le, "capture launch");
    }
    if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
    cudaGraphExec_t x = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&x, g, 0);
    if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ie, "cudaGraphInstantiate");
    }
    net->graph = g;
    net->exec = x;
    net->window = window_steps;
    return N2B_OK;
}

int n2b_replay(n2b_net *net, int64_t n_windows, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    if (!net->exec) return fail(N2B_ESTATE, "no captured window: call n2b_capture first");
    if (n_windows < 0) return fail(N2B_EINVAL, "n_windows < 0");
    N2B_CUDA(cudaSetDevice(net->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int64_t k = 0; k < n_windows; ++k) N2B_CUDA(cudaGraphLaunch(net->exec, s));
    return N2B_OK;
}

int n2b_set_step(n2b_net *net, int64_t step, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    if (step < 0) return fail(N2B_EINVAL, "step < 0");
    N2B_CUDA(cudaSetDevice(net->device));
    n2b::set_step_kernel<<<1, 1, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<long long *>(net->ws + net->L.step), step, reinterpret_cast<int32_t *>(net->ws + net->L.item_count));
    N2B_CUDA(cudaGetLastError());
    return N2B_OK;
}

int n2b_record(n2b_net *net, int64_t step0, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    N2B_CUDA(cudaSetDevice(net->device));
    n2b::set_kernel<<<1, 1, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<long long *>(net->ws + net->L.rec0), step0);
    N2B_CUDA(cudaGetLastError());
    return N2B_OK;
}

int n2b_status(n2b_net *net, int32_t *words, int32_t n_words, void *stream) {
    DeviceGuard guard;
    if (!net || !words || n_words < 0) return fail(N2B_EINVAL, "bad arguments");
    N2B_CUDA(cudaSetDevice(net->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int32_t host[N2B_ERR_WORDS];
    N2B_CUDA(cudaMemcpyAsync(host, net->ws + net->L.err, sizeof(host), cudaMemcpyDeviceToHost, s));
    N2B_CUDA(cudaStreamSynchronize(s));
    for (int32_t k = 0; k < n_words && k < N2B_ERR_WORDS; ++k) words[k] = host[k];
    return N2B_OK;
}

int n2b_counters(n2b_net *net, uint64_t *out, int32_t n_out, void *stream) {
    DeviceGuard guard;
    if (!net || !out || n_out < 0) return fail(N2B_EINVAL, "bad arguments");
    N2B_CUDA(cudaSetDevice(net->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    std::vector<unsigned long long> host(2 + net->n_pops);
    N2B_CUDA(cudaMemcpyAsync(host.data(), net->ws + net->L.counters, sizeof(unsigned long long) * host.size(),
                             cudaMemcpyDeviceToHost, s));
    N2B_CUDA(cudaStreamSynchronize(s));
    for (int32_t k = 0; k < n_out && k < (int32_t)host.size(); ++k) out[k] = host[k];
    return N2B_OK;
}

int n2b_reset_counters(n2b_net *net, void *stream) {
    DeviceGuard guard;
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    N2B_CUDA(cudaSetDevice(net->device));
    n2b::zero_kernel<<<1, 64, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<int32_t *>(net->ws + net->L.err), N2B_ERR_WORDS,
        reinterpret_cast<unsigned long long *>(net->ws + net->L.counters), 2 + net->n_pops);
    N2B_CUDA(cudaMemsetAsync(net->ws + net->L.barrier, 0, sizeof(unsigned) * n2b::BAR_WORDS,
                             reinterpret_cast<cudaStream_t>(stream)));
    N2B_CUDA(cudaGetLastError());
    return N2B_OK;
}

#ifdef N2B_TRACE
// Trace builds only (not part of the C ABI): phase stamps of the next persistent window's first `steps` steps
// into trace[steps][grid][TRACE_PHASES] (device memory).
int n2b_trace(n2b_net *net, unsigned long long *trace, int32_t steps, int32_t *grid) {
    if (!net) return fail(N2B_EINVAL, "net is NULL");
    net->args.trace = trace;
    net->args.trace_steps = steps;
    if (grid) *grid = net->grid;
    return N2B_OK;
}
#endif

int n2b_destroy(n2b_net *net) {
    DeviceGuard guard;
    if (!net) return N2B_OK;
    cudaSetDevice(net->device);
    drop_graph(net);
    delete net;
    return N2B_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------------------------
// n2b_run_static: the same step kernels with their workspace in a fixed device array of this library, for callers
// that cannot allocate device memory (an engine whose own pool holds the GPU's memory, code that must not take
// the device-wide synchronisation of cudaMalloc / cudaFree). The array is the one workspace of every such call on
// a device; each call resets what must start at zero (item counts, error words, counters, barrier) through
// n2b_create's initialisation, so calls whose work overlaps on the GPU race.

static __device__ __align__(256) unsigned char g_static_scratch[N2B_STATIC_SCRATCH_BYTES];

namespace {

// The array's device address on the current device. In host code `g_static_scratch` names a host-side stand-in,
// never the device copy, so the address is asked of the runtime -- on every call: the call is cheap next to
// n2b_create's synchronisations, and an address kept from an earlier call would be stale after a
// cudaDeviceReset (the next primary context maps the array elsewhere).
int static_scratch(void **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_scratch)");
    if (!p || (reinterpret_cast<uintptr_t>(p) & 255) != 0) return fail(N2B_ECUDA, "static scratch misaligned");
    *out = p;
    return N2B_OK;
}

// The far links of step n - 1 (the work list the step kernel of step n would deliver), with no neuron update:
// what is left of a run that stops after step n - 1.
template <int NPB, bool INL>
__global__ void __launch_bounds__(NPB, 2) drain_kernel(const __grid_constant__ n2b::StepArgs a) {
    // a persistent window that gave up at a grid barrier may have left its last step's tiles undone: its work
    // list is then incomplete, and nothing of it is delivered (error word 4 reports the stop)
    if (*(volatile unsigned *)(a.barrier + n2b::BAR_ABORT)) return;
    __shared__ n2b::SConn s_tab[n2b::SMEM_CONNS];
    const n2b::SConn *s_conn = n2b::fill_conns<INL>(a, s_tab, a.n_push);
    __syncthreads();
    n2b::far_phase<NPB, INL, 2>(a, *a.step, s_conn, n2b::far_count(a, *a.step - 1));
}

template <bool INL>
cudaError_t launch_drain(n2b_net *net, cudaStream_t s) {
    const int grid = std::max(net->grid, 1);
    switch (net->block) {
        case 64: drain_kernel<64, INL><<<grid, 64, 0, s>>>(net->args); break;
        case 256: drain_kernel<256, INL><<<grid, 256, 0, s>>>(net->args); break;
        default: drain_kernel<128, INL><<<grid, 128, 0, s>>>(net->args); break;
    }
    return cudaGetLastError();
}

}  // namespace

extern "C" int n2b_run_static(const n2b_population *pops, int32_t n_pops, const n2b_connection *conns,
                              int32_t n_conns, const n2b_options *opt, int64_t step0, int64_t n_steps,
                              int32_t *status, void *stream) {
    if (step0 < 0) return fail(N2B_EINVAL, "step0 < 0");
    if (n_steps < 0 || n_steps > (int64_t)1 << 30) return fail(N2B_EINVAL, "n_steps out of range");
    size_t need = 0;
    int rc = n2b_workspace_bytes(pops, n_pops, conns, n_conns, opt, &need);
    if (rc) return rc;
    if (need > N2B_STATIC_SCRATCH_BYTES)
        return fail(N2B_ESPACE, "n2b_run_static: the network needs " + std::to_string(need) +
                                    " bytes of workspace, the static scratch holds " +
                                    std::to_string((size_t)N2B_STATIC_SCRATCH_BYTES) +
                                    " (use n2b_create with a workspace of the caller's)");
    DeviceGuard guard;
    const int device = opt ? opt->device : 0;
    N2B_CUDA(cudaSetDevice(device));
    void *ws = nullptr;
    rc = static_scratch(&ws);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    n2b_net *net = nullptr;
    rc = n2b_create(pops, n_pops, conns, n_conns, opt, ws, N2B_STATIC_SCRATCH_BYTES, stream, &net);
    if (rc) return rc;
    rc = n2b_set_step(net, step0, stream);
    if (!rc) rc = n2b_record(net, step0, stream);
    if (!rc) rc = n2b_step(net, n_steps, stream);
    if (!rc && n_steps > 0 && net->L.n_tiles > 0) {
        cudaError_t e = net->inl ? launch_drain<true>(net, s) : launch_drain<false>(net, s);
        if (e != cudaSuccess) rc = cuda_fail(e, "drain launch");
    }
    if (!rc && status) {
        int32_t host[N2B_ERR_WORDS];
        cudaError_t e = cudaMemcpyAsync(host, net->ws + net->L.err, sizeof(host), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(e, "status copy");
        else
            for (int k = 0; k < N2B_ERR_WORDS; ++k) status[k] = host[k];
    }
    n2b_destroy(net);
    return rc;
}
