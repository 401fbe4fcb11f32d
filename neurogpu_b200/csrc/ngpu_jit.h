// Runtime specialisation of the advance kernels (host side).
//
// The ahead-of-time advance kernels run every node's channel code on its
// runtime mechanism mask (node_classes.cuh).  For a model in FP32 the library
// generates a small source that instantiates the same kernel bodies with the
// model's own masks as compile-time classes, compiles it with NVRTC for the
// device's architecture, and loads it with the runtime's library API
// (cudaLibraryLoadData).  This is the runtime form of what the reference does
// per model ahead of time: generate the model's channel code and rebuild the
// simulator around it.
//
// NVRTC is loaded with dlopen, so the library has no link-time dependency on
// it.  Compiled images are kept for the life of the process (per mask set)
// and on disk, keyed by a hash of the full source, the options and the NVRTC
// version, under $NGPU_JIT_CACHE or $HOME/.cache/neurogpu_b200.  When NVRTC
// is missing or a compile fails, callers keep the ahead-of-time kernels (the
// generic channel code); NGPU_JIT=0 in the environment selects them too.
// Mechanism sets generated from NMODL files (ngpu_mechset_define) exist only
// as source and always run through this path, in FP32 and FP64.
#pragma once
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "jit_sources.inc"  // generated by _build.py: kJitFiles (the kernel headers' text)

namespace ngpu_jit {

// Parameters compiled in as constants: (index in the mechanism set, value).
using Folds = std::vector<std::pair<int, float>>;

// The literal of a float, exact (hexadecimal).
inline std::string float_literal(float v) {
    char buf[64];
    std::snprintf(buf, sizeof buf, "%af", (double)v);
    return buf;
}

struct Module {
    int mechset = 0;
    bool fp64 = false;
    bool prefetch = true;                   // channel-pass L2 prefetch compiled in (NGPU_CH_PREFETCH)
    bool complete = false;                  // the masks cover every node: no generic path (NGPU_CLASSES_COMPLETE)
    bool ti = false;                        // the thread-item layout's advance kernel compiled in
    int adv_warps = 8;                      // the advance kernels' CTA size bound (warps)
    int adv_ctas = 3;                       // ... and CTAs per SM they are compiled for (above 8 warps)
    std::vector<uint32_t> masks;            // class k runs the code for masks[k]
    cudaLibrary_t lib = nullptr;
    cudaKernel_t init = nullptr;           // (SimArgs<R>)
    cudaKernel_t advance = nullptr;        // (SimArgs<R>, int t0, int n_steps)
    cudaKernel_t batch_init = nullptr;     // (BatchArgs<R>)
    cudaKernel_t batch_advance = nullptr;  // (BatchArgs<R>, int t0, int n_steps)
    cudaKernel_t advance_ti = nullptr;     // (SimArgs<R>, int t0, int n_steps), thread-item layout
};

struct Nvrtc {
    bool ok = false;
    decltype(&::nvrtcVersion) version = nullptr;
    decltype(&::nvrtcCreateProgram) create = nullptr;
    decltype(&::nvrtcCompileProgram) compile = nullptr;
    decltype(&::nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&::nvrtcGetProgramLog) log = nullptr;
    decltype(&::nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&::nvrtcGetCUBIN) cubin = nullptr;
    decltype(&::nvrtcDestroyProgram) destroy = nullptr;
};

inline std::mutex& mu() {
    static std::mutex m;
    return m;
}
inline std::string& last_log() {
    static std::string s;
    return s;
}

inline const Nvrtc& nvrtc() {
    static Nvrtc n = [] {
        Nvrtc r;
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        void* h = nullptr;
        for (const char* nm : names)
            if ((h = dlopen(nm, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) {
            last_log() = "NVRTC not found (libnvrtc.so.12)";
            return r;
        }
#define NGPU_SYM(field, name) r.field = (decltype(r.field))dlsym(h, name)
        NGPU_SYM(version, "nvrtcVersion");
        NGPU_SYM(create, "nvrtcCreateProgram");
        NGPU_SYM(compile, "nvrtcCompileProgram");
        NGPU_SYM(log_size, "nvrtcGetProgramLogSize");
        NGPU_SYM(log, "nvrtcGetProgramLog");
        NGPU_SYM(cubin_size, "nvrtcGetCUBINSize");
        NGPU_SYM(cubin, "nvrtcGetCUBIN");
        NGPU_SYM(destroy, "nvrtcDestroyProgram");
#undef NGPU_SYM
        r.ok = r.version && r.create && r.compile && r.log_size && r.log && r.cubin_size && r.cubin && r.destroy;
        if (!r.ok) last_log() = "NVRTC is missing entry points";
        return r;
    }();
    return n;
}

inline bool enabled() {
    const char* e = std::getenv("NGPU_JIT");
    return !(e && e[0] == '0');
}

// The generated translation unit: the init and advance kernels (single and
// batch) over `masks`.  ms: the kernel template's mechanism set (0 TTPC,
// 1 Mainen, 2 a generated set, whose channel code comes in as the extra
// header ngpu_generated.cuh).  prefetch: the channel pass's L2 prefetch.
// ti: also the thread-item layout's advance kernel.
// adv_warps: the advance kernels are bounded for CTAs of up to this many
// warps; above 8, for adv_ctas CTAs per SM (3 CTAs: 10 warps 64 registers,
// 12: 56, 16: 40; 1 CTA, for batches of at most one CTA per SM: 16 warps
// 128 registers).
inline std::string source(int ms, bool fp64, const std::vector<uint32_t>& masks, bool prefetch = true,
                          const Folds& folds = {}, bool complete = false, bool ti = false, int adv_warps = 8,
                          int adv_ctas = 3) {
    std::string list;
    for (size_t k = 0; k < masks.size(); ++k) list += (k ? ", " : "") + std::to_string(masks[k]) + "u";
    const std::string m = std::to_string(ms);
    const std::string R = fp64 ? "double" : "float";
    const std::string lb = adv_warps > 8
                               ? "__launch_bounds__(" + std::to_string(32 * adv_warps) + ", " +
                                     std::to_string(adv_ctas) + ")"
                               : "__launch_bounds__(ngpu::kLanes * ngpu::kMaxWarps, NGPU_ADV_MIN_BLOCKS)";
    std::string fold;
    if (!folds.empty()) {
        fold = "#include \"param_fold.cuh\"\nnamespace ngpu {\n";
        for (const auto& f : folds)
            fold += "template <> struct ParamFold<" + std::to_string(f.first) +
                    "> { static constexpr bool on = true; static constexpr float v = " + float_literal(f.second) +
                    "; };\n";
        fold += "}\n";
    }
    return std::string(ms == 2 ? "#define NGPU_GENERATED_NODE 1\n" : "") +
           std::string(prefetch ? "" : "#define NGPU_CH_PREFETCH 0\n") +
           std::string(adv_warps > 8 && adv_ctas == 1 ? "#define NGPU_CH_AHEAD 0\n" : "") +
           std::string(complete ? "#define NGPU_CLASSES_COMPLETE 1\n" : "") + fold +
           "#include \"sim_kernels.cuh\"\n"
           "using JitClasses = ngpu::MaskList<" + list + ">;\n"
           "extern \"C\" __global__ void __launch_bounds__(ngpu::kLanes * ngpu::kMaxWarps)\n"
           "ngpu_jit_init(ngpu::SimArgs<" + R + "> A) {\n"
           "    __shared__ int ctr;\n"
           "    ngpu::init_body<" + R + ", " + m + ">(A, blockIdx.x, &ctr);\n"
           "}\n"
           "extern \"C\" __global__ void " + lb + "\n"
           "ngpu_jit_advance(ngpu::SimArgs<" + R + "> A, int t0, int n_steps) {\n"
           "    extern __shared__ __align__(128) char smem[];\n"
           "    __shared__ int ctr[2];\n"
           "    ngpu::advance_body<" + R + ", " + m + ", JitClasses>(A, blockIdx.x, t0, n_steps, smem, ctr);\n"
           "}\n"
           "extern \"C\" __global__ void __launch_bounds__(ngpu::kLanes * ngpu::kMaxWarps)\n"
           "ngpu_jit_batch_init(const __grid_constant__ ngpu::BatchArgs<" + R + "> B) {\n"
           "    __shared__ int ctr;\n"
           "    const int k = ngpu::batch_member(B.cta0, B.n);\n"
           "    ngpu::init_body<" + R + ", " + m + ">(B.sim[k], blockIdx.x - B.cta0[k], &ctr);\n"
           "}\n"
           "extern \"C\" __global__ void " + lb + "\n"
           "ngpu_jit_batch_advance(const __grid_constant__ ngpu::BatchArgs<" + R + "> B, int t0, int n_steps) {\n"
           "    extern __shared__ __align__(128) char smem[];\n"
           "    __shared__ int ctr[2];\n"
           "    const int k = ngpu::batch_member(B.cta0, B.n);\n"
           "    ngpu::advance_body<" + R + ", " + m + ", JitClasses>(B.sim[k], blockIdx.x - B.cta0[k], t0, n_steps,\n"
           "                                                   smem, ctr);\n"
           "}\n" +
           (ti ? "extern \"C\" __global__ void __launch_bounds__(ngpu::kLanes * ngpu::kMaxWarps, NGPU_TI_MIN_BLOCKS)\n"
                 "ngpu_jit_advance_ti(ngpu::SimArgs<" + R + "> A, int t0, int n_steps) {\n"
                 "    extern __shared__ __align__(128) char smem[];\n"
                 "    __shared__ int q[2 * ngpu::kMaxWarps];\n"
                 "    ngpu::advance_body_ti<" + R + ", " + m + ", JitClasses>(A, t0, n_steps, smem, q);\n"
                 "}\n"
               : std::string());
}

inline uint64_t fnv1a(uint64_t h, const std::string& s) {
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

inline std::string cache_dir() {
    if (const char* d = std::getenv("NGPU_JIT_CACHE")) return d;
    if (const char* h = std::getenv("HOME")) return std::string(h) + "/.cache/neurogpu_b200";
    return "";
}

// NVRTC compile of the kernels over `masks` for sm_<arch> (e.g. "100a"),
// through the on-disk cache.  Touches no device.  generated: the channel
// code of a generated mechanism set (ms 2), or nullptr.
inline bool build_cubin(int ms, bool fp64, const std::vector<uint32_t>& masks, const std::string* generated,
                        const std::string& arch, std::vector<char>* out, std::string* err, bool prefetch = true,
                        const Folds& folds = {}, bool complete = false, bool ti = false, int adv_warps = 8,
                        int adv_ctas = 3) {
    const Nvrtc& nv = nvrtc();
    if (!nv.ok) {
        *err = last_log();
        return false;
    }
    const std::string src = source(ms, fp64, masks, prefetch, folds, complete, ti, adv_warps, adv_ctas);
    std::vector<std::string> opt_s = {"--gpu-architecture=sm_" + arch, "-std=c++17",
                                      "-lineinfo"};
    int vmaj = 0, vmin = 0;
    nv.version(&vmaj, &vmin);
    uint64_t h = 1469598103934665603ull;
    h = fnv1a(h, src);
    for (const auto& o : opt_s) h = fnv1a(h, o);
    h = fnv1a(h, std::to_string(vmaj) + "." + std::to_string(vmin));
    const int n_hdr = kJitFileCount + (generated ? 1 : 0);
    std::vector<std::string> hdr_text(n_hdr);
    std::vector<const char*> hdr_src(n_hdr), hdr_name(n_hdr);
    for (int f = 0; f < kJitFileCount; ++f) {
        for (int c = 0; c < kJitFiles[f].n_chunks; ++c) hdr_text[f] += kJitFiles[f].chunks[c];
        hdr_src[f] = hdr_text[f].c_str();
        hdr_name[f] = kJitFiles[f].name;
        h = fnv1a(h, hdr_text[f]);
    }
    if (generated) {
        hdr_text[kJitFileCount] = *generated;
        hdr_src[kJitFileCount] = hdr_text[kJitFileCount].c_str();
        hdr_name[kJitFileCount] = "ngpu_generated.cuh";
        h = fnv1a(h, *generated);
    }
    char hex[17];
    snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)h);
    if (const char* dump = std::getenv("NGPU_JIT_DUMP")) {
        // the translation unit (and a generated set's header) as compiled,
        // for offline inspection with nvcc (register use, spills)
        const std::string base = std::string(dump) + "/" + hex;
        if (FILE* f = fopen((base + ".cu").c_str(), "wb")) {
            fwrite(src.data(), 1, src.size(), f);
            fclose(f);
        }
        if (generated)
            if (FILE* f = fopen((base + "_ngpu_generated.cuh").c_str(), "wb")) {
                fwrite(generated->data(), 1, generated->size(), f);
                fclose(f);
            }
    }
    const std::string dir = cache_dir();
    const std::string path = dir.empty() ? "" : dir + "/" + hex + ".cubin";
    if (!path.empty()) {
        if (FILE* f = fopen(path.c_str(), "rb")) {
            fseek(f, 0, SEEK_END);
            const long n = ftell(f);
            fseek(f, 0, SEEK_SET);
            out->resize(n > 0 ? (size_t)n : 0);
            const bool ok = n > 0 && fread(out->data(), 1, (size_t)n, f) == (size_t)n;
            fclose(f);
            if (ok) return true;
        }
    }
    nvrtcProgram prog = nullptr;
    if (nv.create(&prog, src.c_str(), "ngpu_jit.cu", n_hdr, hdr_src.data(), hdr_name.data()) !=
        NVRTC_SUCCESS) {
        *err = "nvrtcCreateProgram failed";
        return false;
    }
    std::vector<const char*> opts;
    for (const auto& o : opt_s) opts.push_back(o.c_str());
    const nvrtcResult rc = nv.compile(prog, (int)opts.size(), opts.data());
    size_t ls = 0;
    nv.log_size(prog, &ls);
    std::string log(ls, '\0');
    if (ls) nv.log(prog, &log[0]);
    if (rc != NVRTC_SUCCESS) {
        *err = "NVRTC compile failed: " + log;
        nv.destroy(&prog);
        return false;
    }
    size_t cs = 0;
    nv.cubin_size(prog, &cs);
    out->resize(cs);
    nv.cubin(prog, out->data());
    nv.destroy(&prog);
    if (!path.empty()) {  // best effort; a cache that cannot be written is skipped
        std::string p;
        for (size_t i = 0; i <= dir.size(); ++i) {
            if (i == dir.size() || dir[i] == '/') {
                if (!p.empty()) mkdir(p.c_str(), 0755);
            }
            if (i < dir.size()) p += dir[i];
        }
        const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
        if (FILE* f = fopen(tmp.c_str(), "wb")) {
            const bool ok = fwrite(out->data(), 1, out->size(), f) == out->size();
            fclose(f);
            if (ok) rename(tmp.c_str(), path.c_str());
            else remove(tmp.c_str());
        }
    }
    return true;
}

// The module for (mechset, precision, masks) on the current device, compiled
// and loaded on first use; nullptr (reason in last_log()) when runtime
// compilation is off or fails.  mechset >= 2 is a generated set whose channel
// code is *generated.  Modules live until the process exits.
inline const Module* module(int mechset, bool fp64, const std::vector<uint32_t>& masks,
                            const std::string* generated, bool prefetch = true, const Folds& folds = {},
                            bool complete = false, bool ti = false, int adv_warps = 8, int adv_ctas = 3) {
    if (!generated && (!enabled() || masks.empty())) return nullptr;
    if (generated && !enabled()) {
        last_log() = "runtime compilation is off (NGPU_JIT=0)";
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu());
    static std::map<std::string, std::unique_ptr<Module>> cache;
    std::string key = std::to_string(mechset) + (fp64 ? "d" : "f") + (prefetch ? "p" : "n") + (complete ? "c" : "g") +
                      (ti ? "t" : "") +
                      (adv_warps > 8 ? "w" + std::to_string(adv_warps) + "x" + std::to_string(adv_ctas) : std::string()) +
                      ":";
    for (uint32_t m : masks) key += std::to_string(m) + ",";
    for (const auto& f : folds) key += ";" + std::to_string(f.first) + "=" + float_literal(f.second);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second.get();
    int dev = 0, maj = 0, min = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&maj, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&min, cudaDevAttrComputeCapabilityMinor, dev) != cudaSuccess) {
        last_log() = "no CUDA device";
        return nullptr;
    }
    if (maj != 10) {
        last_log() = "runtime compilation targets sm_100a only";
        cache[key] = nullptr;
        return nullptr;
    }
    std::vector<char> cubin;
    std::string err;
    const std::string arch = std::to_string(maj) + std::to_string(min) + "a";
    if (!build_cubin(generated ? 2 : mechset, fp64, masks, generated, arch, &cubin, &err, prefetch, folds,
                     complete, ti, adv_warps, adv_ctas)) {
        last_log() = err;
        cache[key] = nullptr;
        return nullptr;
    }
    auto mod = std::make_unique<Module>();
    mod->mechset = mechset;
    mod->fp64 = fp64;
    mod->prefetch = prefetch;
    mod->complete = complete;
    mod->ti = ti;
    mod->adv_warps = adv_warps;
    mod->adv_ctas = adv_ctas;
    mod->masks = masks;
    cudaError_t e = cudaLibraryLoadData(&mod->lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->init, mod->lib, "ngpu_jit_init");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->advance, mod->lib, "ngpu_jit_advance");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->batch_init, mod->lib, "ngpu_jit_batch_init");
    if (e == cudaSuccess) e = cudaLibraryGetKernel(&mod->batch_advance, mod->lib, "ngpu_jit_batch_advance");
    if (e == cudaSuccess && ti) e = cudaLibraryGetKernel(&mod->advance_ti, mod->lib, "ngpu_jit_advance_ti");
    if (e != cudaSuccess) {
        last_log() = std::string("loading the compiled kernels: ") + cudaGetErrorString(e);
        cudaGetLastError();
        cache[key] = nullptr;
        return nullptr;
    }
    const Module* p = mod.get();
    cache[key] = std::move(mod);
    return p;
}

// The masks to compile for a set of nodes: the distinct masks, at most
// kMaxClasses of them (those carrying the most nodes), in ascending order.
inline std::vector<uint32_t> pick_masks(const std::vector<uint32_t>& node_masks, int max_classes) {
    std::map<uint32_t, long> count;
    for (uint32_t m : node_masks) count[m]++;
    std::vector<std::pair<long, uint32_t>> by;
    for (const auto& kv : count) by.push_back({-kv.second, kv.first});
    std::sort(by.begin(), by.end());
    std::vector<uint32_t> out;
    for (size_t k = 0; k < by.size() && (int)k < max_classes; ++k) out.push_back(by[k].second);
    std::sort(out.begin(), out.end());
    return out;
}

inline int class_of(const Module* mod, uint32_t mask, int generic) {
    if (!mod) return generic;
    for (size_t k = 0; k < mod->masks.size(); ++k)
        if (mod->masks[k] == mask) return (int)k;
    return generic;
}

}  // namespace ngpu_jit
