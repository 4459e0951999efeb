// Run-time compiled operators (paradmm_gpu_register_op_source): the generic
// engine's X phase for factors whose operator the caller gave as device
// source.  The reference GPU back-end calls user __device__ operators
// through device function pointers (core/paradmm-gpu.cu:23-47); here the
// caller's source is compiled once with NVRTC into a kernel that calls the
// operators directly, for the device's architecture, in FP64 without FMA
// contraction (as generic_kernels.cu is built, so an operator written like
// its host twin rounds like it).  NVRTC is loaded with dlopen when first
// needed; compiled kernels are cached for the life of the process.
#include <dlfcn.h>
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "paradmm_gpu.h"

namespace {

typedef int nvrtcResult_t;
typedef struct _nvrtcProgram *nvrtcProgram_t;
struct Nvrtc {
    void *so = nullptr;
    nvrtcResult_t (*create)(nvrtcProgram_t *, const char *, const char *, int, const char *const *, const char *const *) = nullptr;
    nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char *const *) = nullptr;
    nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t *) = nullptr;
    nvrtcResult_t (*log)(nvrtcProgram_t, char *) = nullptr;
    nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t *) = nullptr;
    nvrtcResult_t (*cubin)(nvrtcProgram_t, char *) = nullptr;
    nvrtcResult_t (*destroy)(nvrtcProgram_t *) = nullptr;
};

std::mutex g_mu;
Nvrtc g_nvrtc;
bool g_tried = false;
std::map<std::string, const void *> g_kernels;  // generated source + arch -> kernel

bool load_nvrtc()
{
    if (g_tried) return g_nvrtc.so != nullptr;
    g_tried = true;
    const char *names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12",
                           "/usr/local/cuda/lib64/libnvrtc.so"};
    for (const char *n : names)
        if ((g_nvrtc.so = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!g_nvrtc.so) return false;
    auto sym = [](const char *n) { return dlsym(g_nvrtc.so, n); };
    g_nvrtc.create = (decltype(g_nvrtc.create))sym("nvrtcCreateProgram");
    g_nvrtc.compile = (decltype(g_nvrtc.compile))sym("nvrtcCompileProgram");
    g_nvrtc.log_size = (decltype(g_nvrtc.log_size))sym("nvrtcGetProgramLogSize");
    g_nvrtc.log = (decltype(g_nvrtc.log))sym("nvrtcGetProgramLog");
    g_nvrtc.cubin_size = (decltype(g_nvrtc.cubin_size))sym("nvrtcGetCUBINSize");
    g_nvrtc.cubin = (decltype(g_nvrtc.cubin))sym("nvrtcGetCUBIN");
    g_nvrtc.destroy = (decltype(g_nvrtc.destroy))sym("nvrtcDestroyProgram");
    if (!g_nvrtc.create || !g_nvrtc.compile || !g_nvrtc.log_size || !g_nvrtc.log || !g_nvrtc.cubin_size ||
        !g_nvrtc.cubin || !g_nvrtc.destroy) {
        dlclose(g_nvrtc.so);
        g_nvrtc.so = nullptr;
        return false;
    }
    return true;
}

std::string generate(const std::vector<std::pair<std::string, std::string>> &ops)
{
    std::string src = "// operators given by the caller\n";
    for (const auto &o : ops) src += o.first + "\n";
    src += R"(
extern "C" __global__ void pdm_user_x(int n_user, const int *f_list, const int *f_uid, const long long *f_e0,
                                      const int *f_nv, const long long *f_poff, unsigned char *params, double *X,
                                      double *N, double *RHOS, double *M, const double *U, int d, int with_m)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n_user; t += gridDim.x * blockDim.x) {
        const int f = f_list[t];
        const long long e0 = f_e0[f];
        const int nv = f_nv[f];
        double *x = X + e0 * d;
        double *n = N + e0 * d;
        double *rh = RHOS + e0;
        void *prm = f_poff[f] >= 0 ? (void *)(params + f_poff[f]) : (void *)0;
        switch (f_uid[f]) {
)";
    for (size_t i = 0; i < ops.size(); ++i)
        src += "        case " + std::to_string(i) + ": " + ops[i].second + "(x, n, rh, nv, d, prm); break;\n";
    src += R"(        default: break;
        }
        if (with_m)
            for (int k = 0; k < nv * d; ++k) M[e0 * d + k] = x[k] + U[e0 * d + k];
    }
}
)";
    return src;
}

}  // namespace

int pdm_user_kernel(const std::vector<std::pair<std::string, std::string>> &ops, int device, const void **kernel)
{
    int major = 0, minor = 0;
    PDM_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    PDM_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
    const std::string arch = "--gpu-architecture=sm_" + std::to_string(major) + std::to_string(minor) + (major >= 9 ? "a" : "");
    const std::string src = generate(ops);
    std::lock_guard<std::mutex> lk(g_mu);
    const std::string key = arch + "\n" + src;
    auto it = g_kernels.find(key);
    if (it != g_kernels.end()) { *kernel = it->second; return PARADMM_OK; }
    if (!load_nvrtc())
        return pdm_set_error(PARADMM_EUNSUPPORTED_OP, "run-time compiled operators need NVRTC (libnvrtc.so.12), which could not be loaded");
    nvrtcProgram_t prog = nullptr;
    if (g_nvrtc.create(&prog, src.c_str(), "paradmm_user_ops.cu", 0, nullptr, nullptr) != 0)
        return pdm_set_error(PARADMM_EINVAL, "nvrtcCreateProgram failed");
    const char *opts[] = {arch.c_str(), "--fmad=false", "--std=c++17"};
    const int crc = g_nvrtc.compile(prog, 3, opts);
    if (crc != 0) {
        size_t n = 0;
        g_nvrtc.log_size(prog, &n);
        std::string log(n, '\0');
        if (n) g_nvrtc.log(prog, &log[0]);
        g_nvrtc.destroy(&prog);
        return pdm_set_error(PARADMM_EINVAL, "operator source does not compile: %.400s", log.c_str());
    }
    size_t n = 0;
    g_nvrtc.cubin_size(prog, &n);
    std::vector<char> cubin(n);
    g_nvrtc.cubin(prog, cubin.data());
    g_nvrtc.destroy(&prog);
    cudaLibrary_t lib = nullptr;
    PDM_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
    cudaKernel_t k = nullptr;
    PDM_CUDA(cudaLibraryGetKernel(&k, lib, "pdm_user_x"));
    g_kernels[key] = (const void *)k;
    *kernel = (const void *)k;
    return PARADMM_OK;
}

cudaError_t pdm_launch_user_x(const void *kernel, const GenDev &D, const GenHost &Gh, int with_m, cudaStream_t s)
{
    int n_user = Gh.n_user, d = D.num_dims;
    const int *fl = Gh.d_user_f, *fu = Gh.d_user_id, *fnv = D.f_nv;
    const long long *fe0 = D.f_e0, *fpo = Gh.d_user_poff;
    unsigned char *prm = Gh.d_user_params;
    double *X = (double *)D.X, *N = (double *)D.N, *R = (double *)D.RHOS, *M = (double *)D.M;
    const double *U = (const double *)D.U;
    void *args[] = {&n_user, &fl, &fu, &fe0, &fnv, &fpo, &prm, &X, &N, &R, &M, &U, &d, &with_m};
    const int th = 128;
    const int grid = (int)std::min<long long>((n_user + th - 1) / th, 4096);
    return cudaLaunchKernel(kernel, dim3(grid > 0 ? grid : 1), dim3(th), args, 0, s);
}
