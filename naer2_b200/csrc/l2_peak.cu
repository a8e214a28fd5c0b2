// l2_peak: the L2 atomic throughput of this GPU, the second roofline of the delivery.
//
// Every synaptic event of the step kernels is one 64-bit reduction (red.global.add.u64, no value returned)
// into an arrival slot that stays in L2. This kernel issues the same instruction at pseudo-random slots of a
// caller's L2-sized array, with nothing else to wait for (slot indices come from a per-thread xorshift32,
// no loads), so its rate is what the L2's atomic units sustain for that pattern. bench.py divides the step
// kernels' events/s by it.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__global__ void red_peak_kernel(unsigned long long *slots, uint32_t mask, int ops) {
    uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 0x9E3779B9u;
    for (int k = 0; k < ops; ++k) {
        x ^= x << 13;
        x ^= x >> 17;
        x ^= x << 5;
        asm volatile("red.global.add.u64 [%0], %1;" ::"l"(slots + (x & mask)), "l"(1ull));
    }
}

}  // namespace

extern "C" {

// slots: n_slots zero-initialised uint64 on the current device, n_slots a power of two.
// grid x block threads each add 1 to `ops` slots (grid * block * ops reductions in all) on `stream`.
// Returns 0, -1 for bad arguments, -2 if the launch failed.
int n2b_red_peak(void *slots, int64_t n_slots, int32_t grid, int32_t block, int32_t ops, void *stream) {
    if (!slots || n_slots <= 0 || (n_slots & (n_slots - 1)) != 0 || n_slots > ((int64_t)1 << 32)) return -1;
    if (grid <= 0 || block <= 0 || block > 1024 || ops < 0) return -1;
    red_peak_kernel<<<grid, block, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<unsigned long long *>(slots), (uint32_t)(n_slots - 1), ops);
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // extern "C"
