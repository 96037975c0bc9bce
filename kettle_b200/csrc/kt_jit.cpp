// kt_jit.cpp — run-time compilation of generated block kernels (NVRTC).
//
// The fused-block planner can emit, for each block, CUDA C++ whose gate
// bodies are straight-line code with every register slot, control slot and
// thread / tile mask a compile-time constant (kt_fused.cu, jit_block_body).
// This file compiles such sources for sm_100a with NVRTC, loads the cubins
// with cudaLibraryLoadData and hands back launchable kernels.  NVRTC is
// opened with dlopen at first use, so the library itself has no link-time
// dependency on it; when it cannot be opened, or a compile fails, the caller
// keeps using the precompiled kernels.
//
// The generated sources include the fused device header; its text (and that
// of the header it includes) is embedded at build time (kt_jit_headers.inc,
// written by kettle_b200/build.py into the build directory).
//
// KT_JIT_CACHE_DIR (unset: off) keeps every compiled cubin in that directory
// (created if missing),
// so another process that generates the same source loads it instead of
// compiling it again.  A file is named by a 64-bit hash of everything the
// cubin depends on (the source, the embedded headers, the compile options and
// NVRTC's version) and carries a second, independent hash of the same and a
// hash of its own bytes; a file that fails either check is compiled again and
// replaced.  Files are written under a temporary name and renamed into place.
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nvrtc.h>

#include "kt_internal.cuh"
#include "kt_jit_headers.inc"

namespace kt
{

namespace
{

struct Nvrtc
{
    void* handle {nullptr};
    decltype(&nvrtcCreateProgram) create {nullptr};
    decltype(&nvrtcCompileProgram) compile {nullptr};
    decltype(&nvrtcGetProgramLogSize) log_size {nullptr};
    decltype(&nvrtcGetProgramLog) log {nullptr};
    decltype(&nvrtcGetCUBINSize) cubin_size {nullptr};
    decltype(&nvrtcGetCUBIN) cubin {nullptr};
    decltype(&nvrtcDestroyProgram) destroy {nullptr};
    decltype(&nvrtcGetErrorString) error_string {nullptr};
    decltype(&nvrtcVersion) version {nullptr};
    bool ok {false};
    std::string why;
};

Nvrtc& nvrtc()
{
    static Nvrtc lib;
    static std::once_flag once;
    std::call_once(once, [] {
        const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", "/usr/local/cuda/lib64/libnvrtc.so.12"};
        for (const char* n : names) {
            lib.handle = dlopen(n, RTLD_NOW | RTLD_LOCAL);
            if (lib.handle != nullptr) {
                break;
            }
        }
        if (lib.handle == nullptr) {
            lib.why = "NVRTC (libnvrtc.so.12) could not be opened";
            return;
        }
        auto sym = [&](const char* s) { return dlsym(lib.handle, s); };
        lib.create = reinterpret_cast<decltype(lib.create)>(sym("nvrtcCreateProgram"));
        lib.compile = reinterpret_cast<decltype(lib.compile)>(sym("nvrtcCompileProgram"));
        lib.log_size = reinterpret_cast<decltype(lib.log_size)>(sym("nvrtcGetProgramLogSize"));
        lib.log = reinterpret_cast<decltype(lib.log)>(sym("nvrtcGetProgramLog"));
        lib.cubin_size = reinterpret_cast<decltype(lib.cubin_size)>(sym("nvrtcGetCUBINSize"));
        lib.cubin = reinterpret_cast<decltype(lib.cubin)>(sym("nvrtcGetCUBIN"));
        lib.destroy = reinterpret_cast<decltype(lib.destroy)>(sym("nvrtcDestroyProgram"));
        lib.error_string = reinterpret_cast<decltype(lib.error_string)>(sym("nvrtcGetErrorString"));
        lib.version = reinterpret_cast<decltype(lib.version)>(sym("nvrtcVersion"));
        lib.ok = lib.create && lib.compile && lib.log_size && lib.log && lib.cubin_size && lib.cubin && lib.destroy &&
                 lib.error_string;
        if (!lib.ok) {
            lib.why = "NVRTC is missing an entry point";
        }
    });
    return lib;
}

constexpr const char* JIT_OPTS[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device", "--fmad=true",
                                   "--extra-device-vectorization", "--ptxas-options=-v"};

std::atomic<int64_t> g_nvrtc_compiles {0};
std::atomic<int64_t> g_disk_hits {0};

// FNV-1a, 64 bits, continued from h
uint64_t fnv1a(const void* data, size_t n, uint64_t h)
{
    const auto* b = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) {
        h = (h ^ b[i]) * 0x100000001b3ULL;
    }
    return h;
}

// the two cache hashes of one source: FNV-1a from two different starting
// values over the same material (source, embedded headers, options, NVRTC
// version)
void cache_keys(const std::string& source, uint64_t& k1, uint64_t& k2)
{
    static const std::string common = [] {
        std::string c;
        for (int i = 0; i < KT_JIT_N_HEADERS; ++i) {
            c += KT_JIT_HEADER_NAMES[i];
            c += '\n';
            c += KT_JIT_HEADER_TEXT[i];
            c += '\0';
        }
        for (const char* o : JIT_OPTS) {
            c += o;
            c += '\0';
        }
        int major = 0, minor = 0;
        if (nvrtc().version != nullptr) {
            nvrtc().version(&major, &minor);
        }
        c += "nvrtc " + std::to_string(major) + "." + std::to_string(minor);
        return c;
    }();
    k1 = fnv1a(source.data(), source.size(), fnv1a(common.data(), common.size(), 0xcbf29ce484222325ULL));
    k2 = fnv1a(source.data(), source.size(), fnv1a(common.data(), common.size(), 0x84222325cbf29ce4ULL));
}

constexpr uint64_t CACHE_MAGIC = 0x3130434a54494a4bULL;  // "KJITJC01"

std::string cache_path(const char* dir, uint64_t k1)
{
    char name[40];
    std::snprintf(name, sizeof(name), "/kt_%016llx.cubin", static_cast<unsigned long long>(k1));
    return std::string(dir) + name;
}

// a cached cubin, or empty
std::vector<char> cache_load(const char* dir, uint64_t k1, uint64_t k2)
{
    std::vector<char> out;
    FILE* f = std::fopen(cache_path(dir, k1).c_str(), "rb");
    if (f == nullptr) {
        return out;
    }
    uint64_t head[4] = {0, 0, 0, 0};  // magic, second key, hash of the cubin, its size
    if (std::fread(head, sizeof(head), 1, f) == 1 && head[0] == CACHE_MAGIC && head[1] == k2 &&
        head[3] > 0 && head[3] < (uint64_t {1} << 30)) {
        out.resize(static_cast<size_t>(head[3]));
        if (std::fread(out.data(), 1, out.size(), f) != out.size() ||
            fnv1a(out.data(), out.size(), 0xcbf29ce484222325ULL) != head[2]) {
            out.clear();
        }
    }
    std::fclose(f);
    return out;
}

// the cache directory and its missing parents (mkdir -p)
void cache_mkdir(const char* dir)
{
    std::string d(dir);
    for (size_t pos = 1; pos <= d.size(); ++pos) {
        if (pos == d.size() || d[pos] == '/') {
            mkdir(d.substr(0, pos).c_str(), 0755);  // an existing directory is fine
        }
    }
}

void cache_store(const char* dir, uint64_t k1, uint64_t k2, const std::vector<char>& cubin)
{
    cache_mkdir(dir);
    const std::string path = cache_path(dir, k1);
    const std::string tmp = path + ".tmp" + std::to_string(static_cast<long long>(getpid())) + "_" +
                            std::to_string(std::hash<std::thread::id> {}(std::this_thread::get_id()));
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (f == nullptr) {
        return;  // an unwritable cache only costs the next process a compile
    }
    const uint64_t head[4] = {CACHE_MAGIC, k2, fnv1a(cubin.data(), cubin.size(), 0xcbf29ce484222325ULL),
                              static_cast<uint64_t>(cubin.size())};
    const bool ok = std::fwrite(head, sizeof(head), 1, f) == 1 &&
                    std::fwrite(cubin.data(), 1, cubin.size(), f) == cubin.size();
    if (std::fclose(f) == 0 && ok) {
        std::rename(tmp.c_str(), path.c_str());
    } else {
        std::remove(tmp.c_str());
    }
}

// one source -> one cubin by NVRTC (empty on failure, with the reason in
// `err`); with `info`, ptxas also reports each kernel's registers and spill
// bytes there
std::vector<char> compile_one_nvrtc(const std::string& source, std::string& err, std::string* info)
{
    Nvrtc& L = nvrtc();
    nvrtcProgram prog = nullptr;
    nvrtcResult r = L.create(&prog, source.c_str(), "kt_jit_blocks.cu", KT_JIT_N_HEADERS, KT_JIT_HEADER_TEXT,
                             KT_JIT_HEADER_NAMES);
    if (r != NVRTC_SUCCESS) {
        err = std::string("nvrtcCreateProgram: ") + L.error_string(r);
        return {};
    }
    g_nvrtc_compiles.fetch_add(1);
    const int n_opts = static_cast<int>(sizeof(JIT_OPTS) / sizeof(JIT_OPTS[0])) - (info != nullptr ? 0 : 1);
    r = L.compile(prog, n_opts, JIT_OPTS);
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        L.log_size(prog, &n);
        std::string log(n, '\0');
        if (n > 0) {
            L.log(prog, &log[0]);
        }
        err = std::string("nvrtcCompileProgram: ") + L.error_string(r) + "\n" + log.substr(0, 2000);
        L.destroy(&prog);
        return {};
    }
    if (info != nullptr) {
        size_t m = 0;
        L.log_size(prog, &m);
        info->assign(m, '\0');
        if (m > 0) {
            L.log(prog, &(*info)[0]);
        }
    }
    size_t n = 0;
    L.cubin_size(prog, &n);
    std::vector<char> out(n);
    if (n > 0) {
        L.cubin(prog, out.data());
    }
    L.destroy(&prog);
    return out;
}

// one source -> one cubin (empty on failure, with the reason in `err`); with
// `info`, ptxas also reports each kernel's registers and spill bytes there
std::vector<char> compile_one(const std::string& source, std::string& err, std::string* info = nullptr)
{
    // KT_JIT_CACHE_DIR: a cubin compiled before from the same material
    const char* cache_dir = std::getenv("KT_JIT_CACHE_DIR");
    const bool cached = cache_dir != nullptr && *cache_dir != '\0' && info == nullptr;
    uint64_t k1 = 0, k2 = 0;
    if (cached) {
        cache_keys(source, k1, k2);
        std::vector<char> hit = cache_load(cache_dir, k1, k2);
        if (!hit.empty()) {
            g_disk_hits.fetch_add(1);
            return hit;
        }
    }
    std::vector<char> out = compile_one_nvrtc(source, err, info);
    if (cached && !out.empty()) {
        cache_store(cache_dir, k1, k2, out);
    }
    return out;
}

}  // namespace

int jit_threads()
{
    // the host threads one process compiles with: its share of the machine
    // when several ranks run on it (LOCAL_WORLD_SIZE, as torchrun sets), at
    // most 16 (each NVRTC instance holds a few hundred MB while it compiles)
    unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    if (const char* lws = std::getenv("LOCAL_WORLD_SIZE")) {
        const int ranks = std::atoi(lws);
        if (ranks > 1) {
            hw = std::max(1u, hw / static_cast<unsigned>(ranks));
        }
    }
    return static_cast<int>(std::min(16u, hw));
}

bool jit_available(std::string* why)
{
    Nvrtc& L = nvrtc();
    if (!L.ok && why != nullptr) {
        *why = L.why;
    }
    return L.ok;
}

namespace
{
std::mutex g_libs_mutex;
std::vector<cudaLibrary_t> g_libs;  // every loaded program, until jit_unload_all
}  // namespace

void jit_cache_stats(int64_t* nvrtc_compiles, int64_t* disk_hits)
{
    *nvrtc_compiles = g_nvrtc_compiles.load();
    *disk_hits = g_disk_hits.load();
}

void jit_unload_all()
{
    std::lock_guard<std::mutex> lock(g_libs_mutex);
    for (cudaLibrary_t lib : g_libs) {
        cudaLibraryUnload(lib);
    }
    g_libs.clear();
}

int32_t jit_compile(const std::vector<std::string>& sources, const std::vector<std::vector<std::string>>& names,
                    std::vector<std::vector<const void*>>& kernels, bool load, std::vector<cudaLibrary_t>* owned)
{
    std::string why;
    if (!jit_available(&why)) {
        set_error(KT_ERR_CUDA, why);
        return KT_ERR_CUDA;
    }
    const size_t n = sources.size();
    // KT_JIT_DUMP_DIR: also write each generated program's source there, and
    // ptxas's register / spill summary of its kernels beside it (for inspection)
    const char* dump_dir = std::getenv("KT_JIT_DUMP_DIR");
    const bool dump = dump_dir != nullptr && *dump_dir != '\0';
    std::vector<std::string> infos(n);
    if (dump) {
        const char* dir = dump_dir;
        for (size_t i = 0; i < n; ++i) {
            const std::string path = std::string(dir) + "/kt_jit_" + std::to_string(i) + ".cu";
            if (FILE* f = std::fopen(path.c_str(), "w")) {
                std::fwrite(sources[i].data(), 1, sources[i].size(), f);
                std::fclose(f);
            }
        }
    }
    std::vector<std::vector<char>> cubins(n);
    std::vector<std::string> errs(n);
    const size_t workers = std::max<size_t>(1, std::min<size_t>(n, static_cast<size_t>(jit_threads())));
    std::vector<std::thread> pool;
    std::mutex m;
    size_t next = 0;
    for (size_t w = 0; w < workers; ++w) {
        pool.emplace_back([&] {
            for (;;) {
                size_t i = 0;
                {
                    std::lock_guard<std::mutex> g(m);
                    if (next >= n) {
                        return;
                    }
                    i = next++;
                }
                cubins[i] = compile_one(sources[i], errs[i], dump ? &infos[i] : nullptr);
            }
        });
    }
    for (auto& th : pool) {
        th.join();
    }
    if (dump) {
        for (size_t i = 0; i < n; ++i) {
            const std::string path = std::string(dump_dir) + "/kt_jit_" + std::to_string(i) + ".log";
            if (FILE* f = std::fopen(path.c_str(), "w")) {
                std::fwrite(infos[i].data(), 1, infos[i].size(), f);
                std::fclose(f);
            }
        }
    }
    kernels.assign(n, {});
    for (size_t i = 0; i < n; ++i) {
        if (cubins[i].empty()) {
            set_error(KT_ERR_CUDA, "run-time compile of a block kernel failed: " + errs[i]);
            return KT_ERR_CUDA;
        }
        if (!load) {
            continue;
        }
        cudaLibrary_t lib = nullptr;
        KT_CUDA(cudaLibraryLoadData(&lib, cubins[i].data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
        if (owned != nullptr) {
            owned->push_back(lib);  // the caller unloads it (jit_unload_all leaves it alone)
        } else {
            std::lock_guard<std::mutex> lock(g_libs_mutex);
            g_libs.push_back(lib);
        }
        for (const auto& name : names[i]) {
            cudaKernel_t k = nullptr;
            KT_CUDA(cudaLibraryGetKernel(&k, lib, name.c_str()));
            kernels[i].push_back(reinterpret_cast<const void*>(k));
        }
    }
    return KT_OK;
}

}  // namespace kt
