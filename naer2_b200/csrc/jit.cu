// n2b_jit_*: run-time compilation of the transpiler's step kernels (include/naer2b.h).
//
// The transpiler (naer2_b200/transpiler) turns a population's Python hooks into CUDA device code spliced into
// a step-kernel template; this file compiles that source with NVRTC for the current device's architecture
// (sm_100a on a B200), loads the image with the runtime's library API and launches the kernel with one
// by-value parameter block. NVRTC is loaded with dlopen on first use, so the library loads (and every other
// entry point works) where NVRTC is absent.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/naer2b.h"

namespace n2b_host {
int set_error(int code, const std::string &msg);
}

struct n2b_jit_kernel {
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kernel = nullptr;
    int device = 0;
};

namespace {

struct Nvrtc {
    void *h = nullptr;
    nvrtcResult (*create)(nvrtcProgram *, const char *, const char *, int, const char *const *, const char *const *);
    nvrtcResult (*compile)(nvrtcProgram, int, const char *const *);
    nvrtcResult (*log_size)(nvrtcProgram, size_t *);
    nvrtcResult (*log)(nvrtcProgram, char *);
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t *);
    nvrtcResult (*cubin)(nvrtcProgram, char *);
    nvrtcResult (*destroy)(nvrtcProgram *);
    const char *(*err)(nvrtcResult);
};

std::mutex g_mu;
Nvrtc g_nvrtc;
bool g_tried = false;

// NVRTC from the loader's path, the toolkit's lib64, or PyTorch's wheel directory (N2B_NVRTC overrides).
int load_nvrtc(Nvrtc **out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_tried) {
        g_tried = true;
        std::vector<std::string> names;
        if (const char *env = getenv("N2B_NVRTC")) names.push_back(env);
        names.push_back("libnvrtc.so.12");
        names.push_back("/usr/local/cuda/lib64/libnvrtc.so.12");
        names.push_back("libnvrtc.so");
        for (const auto &n : names) {
            g_nvrtc.h = dlopen(n.c_str(), RTLD_NOW | RTLD_LOCAL);
            if (g_nvrtc.h) break;
        }
        if (g_nvrtc.h) {
            auto sym = [](const char *s) { return dlsym(g_nvrtc.h, s); };
            g_nvrtc.create = reinterpret_cast<decltype(g_nvrtc.create)>(sym("nvrtcCreateProgram"));
            g_nvrtc.compile = reinterpret_cast<decltype(g_nvrtc.compile)>(sym("nvrtcCompileProgram"));
            g_nvrtc.log_size = reinterpret_cast<decltype(g_nvrtc.log_size)>(sym("nvrtcGetProgramLogSize"));
            g_nvrtc.log = reinterpret_cast<decltype(g_nvrtc.log)>(sym("nvrtcGetProgramLog"));
            g_nvrtc.cubin_size = reinterpret_cast<decltype(g_nvrtc.cubin_size)>(sym("nvrtcGetCUBINSize"));
            g_nvrtc.cubin = reinterpret_cast<decltype(g_nvrtc.cubin)>(sym("nvrtcGetCUBIN"));
            g_nvrtc.destroy = reinterpret_cast<decltype(g_nvrtc.destroy)>(sym("nvrtcDestroyProgram"));
            g_nvrtc.err = reinterpret_cast<decltype(g_nvrtc.err)>(sym("nvrtcGetErrorString"));
            if (!g_nvrtc.create || !g_nvrtc.compile || !g_nvrtc.log_size || !g_nvrtc.log || !g_nvrtc.cubin_size ||
                !g_nvrtc.cubin || !g_nvrtc.destroy || !g_nvrtc.err) {
                dlclose(g_nvrtc.h);
                g_nvrtc.h = nullptr;
            }
        }
    }
    if (!g_nvrtc.h) return n2b_host::set_error(N2B_ECUDA, "NVRTC (libnvrtc.so.12) could not be loaded");
    *out = &g_nvrtc;
    return N2B_OK;
}

}  // namespace

// The calling thread's current device, put back when an entry point returns.
struct JitDeviceGuard {
    int prev = -1;
    JitDeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~JitDeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

extern "C" {

int n2b_jit_compile(const char *source, const char *kernel_name, const char *const *options, int32_t n_options,
                    int32_t device, n2b_jit_kernel **out) {
    if (!source || !kernel_name || !out || n_options < 0 || (n_options > 0 && !options))
        return n2b_host::set_error(N2B_EINVAL, "bad arguments");
    *out = nullptr;
    Nvrtc *nv = nullptr;
    int rc = load_nvrtc(&nv);
    if (rc) return rc;
    JitDeviceGuard guard;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return n2b_host::set_error(N2B_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    // the arch-specific target (sm_100a on a B200): the templates may use its features
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(major * 10 + minor) + (major >= 9 ? "a" : "");
    std::vector<const char *> opts = {arch.c_str(), "-std=c++17", "--fmad=false", "-default-device"};
    for (int32_t k = 0; k < n_options; ++k) opts.push_back(options[k]);
    nvrtcProgram prog = nullptr;
    nvrtcResult r = nv->create(&prog, source, "n2b_jit.cu", 0, nullptr, nullptr);
    if (r != NVRTC_SUCCESS) return n2b_host::set_error(N2B_ECUDA, std::string("nvrtcCreateProgram: ") + nv->err(r));
    r = nv->compile(prog, (int)opts.size(), opts.data());
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nv->log_size(prog, &n);
        std::string log(n, '\0');
        if (n) nv->log(prog, &log[0]);
        nv->destroy(&prog);
        return n2b_host::set_error(N2B_EINVAL, std::string("NVRTC compile failed: ") + log);
    }
    size_t n = 0;
    nv->cubin_size(prog, &n);
    std::vector<char> image(n);
    if (n) nv->cubin(prog, image.data());
    nv->destroy(&prog);
    if (!n) return n2b_host::set_error(N2B_ECUDA, "NVRTC returned no device image");
    n2b_jit_kernel *k = new n2b_jit_kernel();
    k->device = device;
    e = cudaLibraryLoadData(&k->lib, image.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&k->kernel, k->lib, kernel_name);
    if (e != cudaSuccess) {
        if (k->lib) cudaLibraryUnload(k->lib);
        delete k;
        return n2b_host::set_error(N2B_ECUDA, std::string("loading the compiled kernel: ") + cudaGetErrorString(e));
    }
    *out = k;
    return N2B_OK;
}

int n2b_jit_launch(n2b_jit_kernel *k, uint32_t grid, uint32_t block, const void *params, size_t params_bytes,
                   void *stream) {
    if (!k || !params || params_bytes == 0 || grid == 0 || block == 0 || block > 1024)
        return n2b_host::set_error(N2B_EINVAL, "bad arguments");
    JitDeviceGuard guard;
    cudaError_t e = cudaSetDevice(k->device);
    if (e == cudaSuccess) {
        void *args[] = {const_cast<void *>(params)};
        e = cudaLaunchKernel(reinterpret_cast<const void *>(k->kernel), dim3(grid), dim3(block), args, 0,
                             reinterpret_cast<cudaStream_t>(stream));
    }
    if (e != cudaSuccess) return n2b_host::set_error(N2B_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
    return N2B_OK;
}

int n2b_jit_launch_window(n2b_jit_kernel *const *kernels, const uint32_t *grids, const uint32_t *blocks,
                          const void *const *params, const size_t *params_bytes, int32_t n_kernels, int64_t step0,
                          int64_t n_steps, double dt, void *stream) {
    if (n_kernels < 0 || n_steps < 0 || (n_kernels > 0 && (!kernels || !grids || !blocks || !params || !params_bytes)))
        return n2b_host::set_error(N2B_EINVAL, "bad arguments");
    std::vector<std::vector<unsigned char>> copy(n_kernels);
    for (int32_t k = 0; k < n_kernels; ++k) {
        if (!kernels[k] || !params[k] || params_bytes[k] < 32 || blocks[k] == 0 || blocks[k] > 1024)
            return n2b_host::set_error(N2B_EINVAL, "bad kernel " + std::to_string(k));
        if (kernels[k]->device != kernels[0]->device)
            return n2b_host::set_error(N2B_EINVAL, "the kernels are loaded on different devices");
        copy[k].assign(static_cast<const unsigned char *>(params[k]),
                       static_cast<const unsigned char *>(params[k]) + params_bytes[k]);
    }
    if (n_kernels == 0 || n_steps == 0) return N2B_OK;
    JitDeviceGuard guard;
    cudaError_t e = cudaSetDevice(kernels[0]->device);
    for (int64_t s = 0; e == cudaSuccess && s < n_steps; ++s) {
        const int64_t n = step0 + s;
        const float t = (float)((double)(n + 1) * dt), t0 = (float)((double)n * dt);
        for (int32_t k = 0; e == cudaSuccess && k < n_kernels; ++k) {
            if (grids[k] == 0) continue;
            unsigned char *P = copy[k].data();
            std::memcpy(P, &n, sizeof(n));
            std::memcpy(P + 24, &t, sizeof(t));
            std::memcpy(P + 28, &t0, sizeof(t0));
            void *args[] = {P};  // (the launch copies the parameter block)
            e = cudaLaunchKernel(reinterpret_cast<const void *>(kernels[k]->kernel), dim3(grids[k]), dim3(blocks[k]),
                                 args, 0, reinterpret_cast<cudaStream_t>(stream));
        }
    }
    if (e != cudaSuccess) return n2b_host::set_error(N2B_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
    return N2B_OK;
}

int n2b_jit_destroy(n2b_jit_kernel *k) {
    if (!k) return N2B_OK;
    JitDeviceGuard guard;
    cudaSetDevice(k->device);
    if (k->lib) cudaLibraryUnload(k->lib);
    delete k;
    return N2B_OK;
}

}  // extern "C"
