// Right-hand sides compiled at run time: C expressions -> a device functor inside
// the fused integrator templates -> NVRTC (sm_100a) -> a module whose kernels run
// the same solve passes as the built-in systems (pb_api.cu:solve_with).
//
// NVRTC is loaded with dlopen and the driver-API calls come from
// cudaGetDriverEntryPoint, so the library links neither libnvrtc nor libcuda.
#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "pb_launch.h"
#include "pybasin_b200.h"

namespace pb {

// ---------------------------------------------------------------------------
// driver API through the runtime's entry-point table
// ---------------------------------------------------------------------------
namespace {

using FnLaunch = CUresult (*)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                              CUstream, void**, void**);
using FnOccupancy = CUresult (*)(int*, CUfunction, int, size_t);
using FnSetAttr = CUresult (*)(CUfunction, CUfunction_attribute, int);
using FnModLoad = CUresult (*)(CUmodule*, const void*);
using FnModGet = CUresult (*)(CUfunction*, CUmodule, const char*);
using FnModUnload = CUresult (*)(CUmodule);

struct Driver {
    FnLaunch launch = nullptr;
    FnOccupancy occupancy = nullptr;
    FnSetAttr set_attr = nullptr;
    FnModLoad mod_load = nullptr;
    FnModGet mod_get = nullptr;
    FnModUnload mod_unload = nullptr;
    bool ok = false;
};

template <class F>
bool entry(const char* name, F* out)
{
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess ||
        !p)
        return false;
    *out = reinterpret_cast<F>(p);
    return true;
}

const Driver& driver()
{
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        d.ok = entry("cuLaunchKernel", &d.launch) &&
               entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", &d.occupancy) &&
               entry("cuFuncSetAttribute", &d.set_attr) && entry("cuModuleLoadData", &d.mod_load) &&
               entry("cuModuleGetFunction", &d.mod_get) && entry("cuModuleUnload", &d.mod_unload);
    });
    return d;
}

cudaError_t from_cu(CUresult r) { return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure; }

// ---------------------------------------------------------------------------
// NVRTC through dlopen
// ---------------------------------------------------------------------------
struct Nvrtc {
    nvrtcResult (*create)(nvrtcProgram*, const char*, const char*, int, const char* const*, const char* const*) =
        nullptr;
    nvrtcResult (*compile)(nvrtcProgram, int, const char* const*) = nullptr;
    nvrtcResult (*log_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*get_log)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*cubin_size)(nvrtcProgram, size_t*) = nullptr;
    nvrtcResult (*get_cubin)(nvrtcProgram, char*) = nullptr;
    nvrtcResult (*add_name)(nvrtcProgram, const char*) = nullptr;
    nvrtcResult (*lowered)(nvrtcProgram, const char*, const char**) = nullptr;
    nvrtcResult (*destroy)(nvrtcProgram*) = nullptr;
    nvrtcResult (*version)(int*, int*) = nullptr;
    bool ok = false;
};

template <class F>
bool sym(void* h, const char* name, F* out)
{
    void* p = dlsym(h, name);
    if (!p) return false;
    *out = reinterpret_cast<F>(p);
    return true;
}

const Nvrtc& nvrtc()
{
    static Nvrtc n;
    static std::once_flag once;
    std::call_once(once, [] {
        std::vector<std::string> cands;
        if (const char* e = std::getenv("PB_NVRTC_LIBRARY")) cands.emplace_back(e);
        if (const char* h = std::getenv("CUDA_HOME")) cands.emplace_back(std::string(h) + "/lib64/libnvrtc.so.12");
        cands.emplace_back("/usr/local/cuda/lib64/libnvrtc.so.12");
        cands.emplace_back("libnvrtc.so.12");
        void* h = nullptr;
        for (const auto& c : cands)
            if ((h = dlopen(c.c_str(), RTLD_NOW | RTLD_LOCAL)) != nullptr) break;
        if (!h) return;
        n.ok = sym(h, "nvrtcCreateProgram", &n.create) && sym(h, "nvrtcCompileProgram", &n.compile) &&
               sym(h, "nvrtcGetProgramLogSize", &n.log_size) && sym(h, "nvrtcGetProgramLog", &n.get_log) &&
               sym(h, "nvrtcGetCUBINSize", &n.cubin_size) && sym(h, "nvrtcGetCUBIN", &n.get_cubin) &&
               sym(h, "nvrtcAddNameExpression", &n.add_name) && sym(h, "nvrtcGetLoweredName", &n.lowered) &&
               sym(h, "nvrtcDestroyProgram", &n.destroy) && sym(h, "nvrtcVersion", &n.version);
    });
    return n;
}

// kernels of one program, in KernelSel order
constexpr int kNumKernels = 6;  // the sampling pass is shared with the built-in systems

std::vector<std::string> kernel_names(int precision)
{
    const std::string s(precision == PB_PREC_FP64 ? "double" : "float");
    return {
        "pb::k_solve_plain<pb::SysUser, " + s + ", false>",
        "pb::k_solve_plain<pb::SysUser, " + s + ", true>",
        "pb::k_solve_queue<pb::SysUser, " + s + ", false, 0>",
        "pb::k_solve_queue<pb::SysUser, " + s + ", true, 0>",
        "pb::k_solve_queue<pb::SysUser, " + s + ", true, 1>",
        "pb::k_solve_queue<pb::SysUser, " + s + ", true, 2>",
    };
}

std::string generate_source(const char* const* rhs, int dim, int n_params, const char* preamble)
{
    std::string src;
    src += "// generated by pb_rhs_compile\n#include \"pb_dopri5.cuh\"\nnamespace pb {\n";
    if (preamble) src += std::string(preamble) + "\n";
    src += "struct SysUser {\n";
    src += "    static constexpr int S = " + std::to_string(dim) + ";\n";
    src += "    static constexpr int NP = " + std::to_string(n_params > 0 ? n_params : 1) + ";\n";
    src += "    static constexpr bool kTime = true;\n    static constexpr bool kExactTime = true;\n";
    src += "    template <class R, class C>\n";
    src += "    __device__ __forceinline__ static void f(const C& clock, const R* y, R* dy, const R* p)\n    {\n";
    src += "        const double t = clock_time(clock);\n        (void)t;\n        (void)p;\n";
    for (int i = 0; i < dim; ++i)
        src += "        dy[" + std::to_string(i) + "] = static_cast<R>(" + std::string(rhs[i]) + ");\n";
    src += "    }\n};\n}  // namespace pb\n";
    return src;
}

uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull)
{
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

void copy_log(const std::string& msg, char* log, int64_t log_bytes)
{
    if (!log || log_bytes <= 0) return;
    const size_t n = msg.size() < static_cast<size_t>(log_bytes - 1) ? msg.size() : static_cast<size_t>(log_bytes - 1);
    std::memcpy(log, msg.data(), n);
    log[n] = '\0';
}

// library directory (for the default include paths)
std::string library_dir()
{
    Dl_info info;
    if (dladdr(reinterpret_cast<void*>(&library_dir), &info) == 0 || !info.dli_fname) return ".";
    std::string p(info.dli_fname);
    const size_t k = p.rfind('/');
    return k == std::string::npos ? "." : p.substr(0, k);
}

bool read_file(const std::string& path, std::string& out)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    out.clear();
    char buf[1 << 16];
    size_t r;
    while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, r);
    std::fclose(f);
    return true;
}

// cache file: "PBRHS1\n", the lowered kernel names one per line, "\n", the cubin
bool read_cache(const std::string& path, std::vector<std::string>& names, std::string& cubin)
{
    std::string data;
    if (!read_file(path, data)) return false;
    size_t pos = data.find('\n');
    if (pos == std::string::npos || data.compare(0, pos, "PBRHS1") != 0) return false;
    names.clear();
    for (int i = 0; i < kNumKernels; ++i) {
        const size_t e = data.find('\n', pos + 1);
        if (e == std::string::npos) return false;
        names.push_back(data.substr(pos + 1, e - pos - 1));
        pos = e;
    }
    if (pos + 2 > data.size() || data[pos + 1] != '\n') return false;
    cubin = data.substr(pos + 2);
    return !cubin.empty();
}

void write_cache(const std::string& path, const std::vector<std::string>& names, const std::string& cubin)
{
    const std::string tmp = path + ".tmp" + std::to_string(static_cast<long long>(reinterpret_cast<intptr_t>(&names)));
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return;
    std::string head = "PBRHS1\n";
    for (const auto& n : names) head += n + "\n";
    head += "\n";
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size() &&
              std::fwrite(cubin.data(), 1, cubin.size(), f) == cubin.size();
    ok = (std::fclose(f) == 0) && ok;
    if (ok)
        std::rename(tmp.c_str(), path.c_str());
    else
        std::remove(tmp.c_str());
}

}  // namespace

cudaError_t drv_launch(void* fn, unsigned grid, unsigned block, unsigned smem, cudaStream_t st, void** argv)
{
    const Driver& d = driver();
    if (!d.ok) return cudaErrorNotSupported;
    return from_cu(d.launch(static_cast<CUfunction>(fn), grid, 1, 1, block, 1, 1, smem, reinterpret_cast<CUstream>(st),
                            argv, nullptr));
}

cudaError_t drv_occupancy(void* fn, int block, int smem, int* blocks_per_sm)
{
    const Driver& d = driver();
    if (!d.ok) return cudaErrorNotSupported;
    return from_cu(d.occupancy(blocks_per_sm, static_cast<CUfunction>(fn), block, static_cast<size_t>(smem)));
}

cudaError_t drv_set_max_smem(void* fn, int bytes)
{
    const Driver& d = driver();
    if (!d.ok) return cudaErrorNotSupported;
    return from_cu(d.set_attr(static_cast<CUfunction>(fn), CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, bytes));
}

}  // namespace pb

struct pb_rhs_program {
    int device;
    int dim;
    int n_params;
    int precision;
    CUmodule module;
    pb::KernelSel k;
};

using namespace pb;

extern "C" {

int pb_rhs_compile(const char* const* rhs, int32_t dim, int32_t n_params, const char* preamble, int32_t precision,
                   const char* const* include_dirs, int32_t n_include_dirs, const char* cache_dir,
                   pb_rhs_program** out, char* log, int64_t log_bytes)
{
    if (out) *out = nullptr;
    if (!rhs || dim < 1 || dim > PB_MAX_USER_DIM || n_params < 0 || n_params > PB_MAX_PARAMS) return PB_EINVAL;
    if (precision != PB_PREC_FP64 && precision != PB_PREC_MIXED) return PB_EINVAL;
    if (n_include_dirs < 0 || (n_include_dirs > 0 && !include_dirs)) return PB_EINVAL;
    for (int i = 0; i < dim; ++i)
        if (!rhs[i] || !rhs[i][0]) return PB_EINVAL;

    const std::string src = generate_source(rhs, dim, n_params, preamble);
    std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-default-device"};
    if (n_include_dirs > 0) {
        for (int i = 0; i < n_include_dirs; ++i) opts.push_back(std::string("-I") + include_dirs[i]);
    } else {
        const std::string lib = library_dir();
        opts.push_back("-I" + lib + "/../csrc");
        opts.push_back("-I" + lib + "/../../include");
    }
    const std::vector<std::string> wanted = kernel_names(precision);

    // the key covers the generated source, the options, the kernels (precision),
    // the NVRTC version and the kernel headers
    const Nvrtc& nv = nvrtc();
    int vmaj = 0, vmin = 0;
    if (nv.ok) nv.version(&vmaj, &vmin);
    std::string keytext = src;
    for (const auto& o : opts) keytext += "\n" + o;
    for (const auto& w : wanted) keytext += "\n" + w;
    // and the kernel headers the program includes, read from the include paths
    for (const char* h : {"pb_dopri5.cuh", "pb_rhs.cuh", "pb_scratch.cuh", "pb_compat.cuh", "pybasin_b200.h"}) {
        for (const auto& o : opts) {
            if (o.compare(0, 2, "-I") != 0) continue;
            std::string text;
            if (read_file(o.substr(2) + "/" + h, text)) {
                keytext += "\n" + text;
                break;
            }
        }
    }
    keytext += "\nnvrtc " + std::to_string(vmaj) + "." + std::to_string(vmin);
    char keyhex[32];
    std::snprintf(keyhex, sizeof keyhex, "%016llx", static_cast<unsigned long long>(fnv1a(keytext)));
    const std::string cache_path = cache_dir ? std::string(cache_dir) + "/pbrhs_" + keyhex + ".bin" : std::string();

    std::vector<std::string> lowered;
    std::string cubin;
    if (!(cache_dir && read_cache(cache_path, lowered, cubin))) {
        if (!nv.ok) {
            copy_log("NVRTC library not found (set PB_NVRTC_LIBRARY)", log, log_bytes);
            return PB_EUNSUPPORTED;
        }
        nvrtcProgram prog;
        if (nv.create(&prog, src.c_str(), "pb_user_rhs.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) return PB_ECOMPILE;
        for (const auto& w : wanted) nv.add_name(prog, w.c_str());
        std::vector<const char*> copt;
        for (const auto& o : opts) copt.push_back(o.c_str());
        const nvrtcResult cr = nv.compile(prog, static_cast<int>(copt.size()), copt.data());
        size_t lsz = 0;
        nv.log_size(prog, &lsz);
        std::string lg(lsz, '\0');
        if (lsz > 0) nv.get_log(prog, &lg[0]);
        copy_log(lg, log, log_bytes);
        if (cr != NVRTC_SUCCESS) {
            nv.destroy(&prog);
            return PB_ECOMPILE;
        }
        size_t csz = 0;
        nv.cubin_size(prog, &csz);
        cubin.assign(csz, '\0');
        if (csz == 0 || nv.get_cubin(prog, &cubin[0]) != NVRTC_SUCCESS) {
            nv.destroy(&prog);
            return PB_ECOMPILE;
        }
        lowered.clear();
        for (const auto& w : wanted) {
            const char* ln = nullptr;
            if (nv.lowered(prog, w.c_str(), &ln) != NVRTC_SUCCESS || !ln) {
                nv.destroy(&prog);
                return PB_ECOMPILE;
            }
            lowered.emplace_back(ln);
        }
        nv.destroy(&prog);
        if (cache_dir) write_cache(cache_path, lowered, cubin);
    }
    if (!out) return PB_SUCCESS;  // compile-ahead: no device needed

    const Driver& d = driver();
    if (!d.ok) return PB_EUNSUPPORTED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return PB_ECUDA;  // primary context
    CUmodule mod = nullptr;
    if (d.mod_load(&mod, cubin.data()) != CUDA_SUCCESS) return PB_ECUDA;
    CUfunction fns[kNumKernels];
    for (int i = 0; i < kNumKernels; ++i)
        if (d.mod_get(&fns[i], mod, lowered[i].c_str()) != CUDA_SUCCESS) {
            d.mod_unload(mod);
            return PB_ECUDA;
        }
    auto* p = new pb_rhs_program;
    p->device = dev;
    p->dim = dim;
    p->n_params = n_params;
    p->precision = precision;
    p->module = mod;
    KFn* slots[kNumKernels] = {&p->k.plain,     &p->k.plain_defer, &p->k.queue,
                               &p->k.queue_defer, &p->k.queue_probe, &p->k.queue_main};
    for (int i = 0; i < kNumKernels; ++i) slots[i]->drv = fns[i];
    p->k.smem_per_thread = 6 * dim * 8 + (PB_MAX_CROSSING + 2) * 4;  // Stats<S>::kBytesPerThread
    *out = p;
    return PB_SUCCESS;
}

int pb_solve_batch_rhs(const pb_rhs_program* prog, const pb_solve_args* args, void* stream)
{
    if (!prog) return PB_EINVAL;
    int v = validate_args(args, true);
    if (v != PB_SUCCESS) return v;
    if (args->dim != prog->dim || args->precision != prog->precision || args->n_params != prog->n_params)
        return PB_EINVALID_ODE;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PB_ECUDA;
    if (dev != prog->device) return PB_EINVAL;  // the module lives on the device it was loaded on
    return solve_with(prog->k, *args, static_cast<cudaStream_t>(stream));
}

int pb_rhs_release(pb_rhs_program* prog)
{
    if (!prog) return PB_SUCCESS;
    const Driver& d = driver();
    int rc = PB_SUCCESS;
    if (prog->module && d.ok && d.mod_unload(prog->module) != CUDA_SUCCESS) rc = PB_ECUDA;
    delete prog;
    return rc;
}

}  // extern "C"
