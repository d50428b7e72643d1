// jit.cpp -- NVRTC compilation, caching and loading of the rule-specialised tick kernels (jit.h).
//
// NVRTC is loaded with dlopen on first use, so the library has no link-time dependency on it;
// when it is missing every key stays on the generic kernel. The kernel sources are the
// library's own device headers, embedded at build time (jit_sources.cpp, generated by
// cave_b200/build.py), so a specialised kernel always matches the library it runs in.
// Compiled cubins are cached on disk under CAVE_JIT_CACHE (default
// $XDG_CACHE_HOME/cave_b200 or ~/.cache/cave_b200; "off" disables the disk cache), named by a
// hash of the sources, the options and the CUDA toolkit version the library was built with.
#include "jit.h"
#include "trace.h"

#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <type_traits>
#include <vector>

namespace cave {

extern const int kJitSourceCount;
extern const char* const kJitSourceNames[];
extern const char* const kJitSourceTexts[];

namespace {

// The translation unit NVRTC compiles: the tick kernel body with the rule as constants.
const char* const kJitUnit = R"cave_unit(
#include "stream_tick.cuh"
#include "stream_tick2.cuh"
namespace cave {
struct JitRule {
    static constexpr bool kFixed = true;
    static constexpr bool kFullRange = CAVE_JIT_MAXCS == 15u;
    __device__ static DeviceRule rule() {
        DeviceRule r{};
        r.maxcs = CAVE_JIT_MAXCS;
        r.flags = CAVE_JIT_NB;
        r.lut_s = CAVE_JIT_LUT_S;
        r.lut_b = CAVE_JIT_LUT_B;
        for (int i = 0; i < 4; i++) r.m[i] = (((CAVE_JIT_MAXCS & 15u) >> i) & 1u) ? 0xFFFFFFFFu : 0u;
        r.alive_ok = CAVE_JIT_MAXCS <= 15u ? 0xFFFFFFFFu : 0u;
        r.nterms = 0;
        return r;
    }
};
}  // namespace cave
#define CAVE_JIT_KERNEL(NAME, COUNT_ZERO, DENSE)                                                           \
    extern "C" __global__ void __launch_bounds__(cave::kJitMaxThreads, 1)                                  \
        NAME(const cave::StreamItem* __restrict__ items, cave::StripSim* sims, uint4* pool, uint32_t sxp_log2, \
             int tick_arg) {                                                                               \
        cave::stream_tick_body<CAVE_JIT_NB, 0, false, cave::JitRule, COUNT_ZERO, DENSE,                     \
                               COUNT_ZERO ? cave::kPopNone : cave::kPopInput, cave::kJitRowsPerThread>(    \
            items, sims, pool, sxp_log2, tick_arg, cave::DeviceRule{});                                    \
    }
CAVE_JIT_KERNEL(cave_stream_tick_jit, true, false)
CAVE_JIT_KERNEL(cave_stream_tick_jit_derived, false, false)
CAVE_JIT_KERNEL(cave_stream_tick_jit_dense, true, true)
CAVE_JIT_KERNEL(cave_stream_tick_jit_dense_derived, false, true)
#define CAVE_JIT_KERNEL2(NAME, FIRST, DENSE)                                                              \
    extern "C" __global__ void __launch_bounds__(cave::kJit2MaxThreads, cave::kJit2CtasPerSm)              \
        NAME(const cave::StreamItem* __restrict__ items, cave::StripSim* sims, uint4* pool, uint32_t sxp_log2, \
             int tick_arg, int src_sel) {                                                                  \
        cave::stream_tick2_body<CAVE_JIT_NB, cave::JitRule, FIRST, DENSE, cave::kJit2RowsPerThread>(       \
            items, sims, pool, sxp_log2, tick_arg, src_sel);                                               \
    }
CAVE_JIT_KERNEL2(cave_stream_tick2_jit_first, true, false)
CAVE_JIT_KERNEL2(cave_stream_tick2_jit, false, false)
CAVE_JIT_KERNEL2(cave_stream_tick2_jit_dense_first, true, true)
CAVE_JIT_KERNEL2(cave_stream_tick2_jit_dense, false, true)
)cave_unit";
const char* const kJitCounting[2] = {"cave_stream_tick_jit", "cave_stream_tick_jit_dense"};
const char* const kJitDerived[2] = {"cave_stream_tick_jit_derived", "cave_stream_tick_jit_dense_derived"};
const char* const kJitPairFirst[2] = {"cave_stream_tick2_jit_first", "cave_stream_tick2_jit_dense_first"};
const char* const kJitPair[2] = {"cave_stream_tick2_jit", "cave_stream_tick2_jit_dense"};

struct Nvrtc {
    bool ok = false;
    std::string why;
    int major = 0, minor = 0;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcGetErrorString) error_string = nullptr;
    decltype(&nvrtcVersion) version = nullptr;
};

Nvrtc load_nvrtc() {
    Nvrtc n;
    std::vector<std::string> names = {"libnvrtc.so.12", "libnvrtc.so"};
    if (const char* h = std::getenv("CUDA_HOME")) names.push_back(std::string(h) + "/lib64/libnvrtc.so.12");
    names.push_back("/usr/local/cuda/lib64/libnvrtc.so.12");
    void* so = nullptr;
    for (const std::string& s : names)
        if ((so = dlopen(s.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
    if (!so) {
        n.why = "NVRTC (libnvrtc.so.12) not found";
        return n;
    }
    bool all = true;
    auto sym = [&](auto& fn, const char* name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(so, name));
        all = all && fn != nullptr;
    };
    sym(n.create, "nvrtcCreateProgram");
    sym(n.compile, "nvrtcCompileProgram");
    sym(n.destroy, "nvrtcDestroyProgram");
    sym(n.log_size, "nvrtcGetProgramLogSize");
    sym(n.log, "nvrtcGetProgramLog");
    sym(n.cubin_size, "nvrtcGetCUBINSize");
    sym(n.cubin, "nvrtcGetCUBIN");
    sym(n.error_string, "nvrtcGetErrorString");
    sym(n.version, "nvrtcVersion");
    if (!all) {
        n.why = "NVRTC lacks an expected entry point";
        return n;
    }
    n.version(&n.major, &n.minor);
    n.ok = true;
    return n;
}

Nvrtc& nvrtc() {
    static Nvrtc n = load_nvrtc();
    return n;
}

// FNV-1a, 64-bit (Fowler, Noll, Vo).
uint64_t fnv1a(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

std::string cache_dir() {
    const char* env = std::getenv("CAVE_JIT_CACHE");
    std::string d;
    if (env) {
        if (!std::strcmp(env, "off") || !*env) return std::string();
        d = env;
    } else if (const char* x = std::getenv("XDG_CACHE_HOME")) {
        d = std::string(x) + "/cave_b200";
    } else if (const char* h = std::getenv("HOME")) {
        d = std::string(h) + "/.cache/cave_b200";
    } else {
        return std::string();
    }
    // create the directory and its parent (best effort; an unusable directory disables the cache)
    const size_t slash = d.find_last_of('/');
    if (slash != std::string::npos && slash > 0) mkdir(d.substr(0, slash).c_str(), 0755);
    mkdir(d.c_str(), 0755);
    return access(d.c_str(), W_OK) == 0 ? d : std::string();
}

std::vector<std::string> options_for(const JitKey& k) {
    char b[4][64];
    std::snprintf(b[0], sizeof b[0], "-DCAVE_JIT_NB=%u", k.nb);
    std::snprintf(b[1], sizeof b[1], "-DCAVE_JIT_MAXCS=%uu", k.maxcs);
    std::snprintf(b[2], sizeof b[2], "-DCAVE_JIT_LUT_S=0x%xu", k.lut_s);
    std::snprintf(b[3], sizeof b[3], "-DCAVE_JIT_LUT_B=0x%xu", k.lut_b);
    // -default-device: the C header's declarations (host functions) are parsed as device ones
    std::vector<std::string> o = {"--gpu-architecture=sm_100a", "-std=c++20", "-default-device", "-lineinfo",
                                  b[0], b[1], b[2], b[3],
                                  "-DCAVE_TICK2_ROWS=" + std::to_string(tick2_geometry().rows_per_thread),
                                  "-DCAVE_TICK2_THREADS=" + std::to_string(tick2_geometry().max_threads),
                                  "-DCAVE_TICK2_CTAS=" + std::to_string(tick2_geometry().ctas_per_sm)};
#ifdef CAVE_CHECKED
    o.push_back("-DCAVE_CHECKED");  // the checked library compiles checked kernels
#endif
    return o;
}

// Compiles the kernel for k (or reads it from the disk cache). No device is touched.
bool compile_cubin(const JitKey& k, std::vector<char>* out, std::string* log) {
    TraceRange trace("jit_compile");
    const std::vector<std::string> opts = options_for(k);
    uint64_t h = fnv1a(kJitUnit, std::strlen(kJitUnit));
    for (int i = 0; i < kJitSourceCount; i++) {
        h = fnv1a(kJitSourceNames[i], std::strlen(kJitSourceNames[i]) + 1, h);
        h = fnv1a(kJitSourceTexts[i], std::strlen(kJitSourceTexts[i]) + 1, h);
    }
    for (const std::string& o : opts) h = fnv1a(o.c_str(), o.size() + 1, h);
    const int toolkit = CUDART_VERSION;  // the toolkit the library was built with
    h = fnv1a(&toolkit, sizeof toolkit, h);
    const std::string dir = cache_dir();
    char fname[64];
    std::snprintf(fname, sizeof fname, "/stream_tick_%016llx.cubin", (unsigned long long)h);
    const std::string path = dir.empty() ? std::string() : dir + fname;
    if (!path.empty()) {
        std::ifstream f(path, std::ios::binary);
        if (f) {
            std::vector<char> data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
            if (!data.empty()) {
                *out = std::move(data);
                return true;
            }
        }
    }
    // NVRTC is loaded only now: a process that finds its kernels in the disk cache never maps it
    Nvrtc& n = nvrtc();
    if (!n.ok) {
        *log = n.why;
        return false;
    }
    nvrtcProgram prog = nullptr;
    nvrtcResult r = n.create(&prog, kJitUnit, "cave_stream_tick_jit.cu", kJitSourceCount, kJitSourceTexts,
                             kJitSourceNames);
    if (r != NVRTC_SUCCESS) {
        *log = std::string("nvrtcCreateProgram: ") + n.error_string(r);
        return false;
    }
    std::vector<const char*> argv;
    for (const std::string& o : opts) argv.push_back(o.c_str());
    r = n.compile(prog, (int)argv.size(), argv.data());
    size_t ls = 0;
    n.log_size(prog, &ls);
    std::string text(ls, '\0');
    if (ls) n.log(prog, text.data());
    while (!text.empty() && text.back() == '\0') text.pop_back();
    size_t cs = 0;
    if (r == NVRTC_SUCCESS) r = n.cubin_size(prog, &cs);
    if (r == NVRTC_SUCCESS && cs) {
        out->resize(cs);
        r = n.cubin(prog, out->data());
    }
    n.destroy(&prog);
    if (r != NVRTC_SUCCESS || cs == 0) {
        *log = std::string("NVRTC: ") + n.error_string(r) + "\n" + text;
        return false;
    }
    *log = text;
    if (!path.empty()) {  // write-then-rename, so readers never see a partial file
        const std::string tmp = path + "." + std::to_string((long)getpid()) + ".tmp";
        std::ofstream f(tmp, std::ios::binary);
        if (f.write(out->data(), (std::streamsize)out->size()) && f.flush()) {
            f.close();
            std::rename(tmp.c_str(), path.c_str());
        } else {
            std::remove(tmp.c_str());
        }
    }
    return true;
}

enum class State { None, Queued, Compiled, Loaded, Failed };
struct Entry {
    State state = State::None;
    std::vector<char> cubin;
    std::string log;
    cudaLibrary_t lib = nullptr;
    JitKernels kern;
};
using Key = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;
Key key_of(const JitKey& k) { return Key{k.nb, k.maxcs, k.lut_s, k.lut_b}; }

// Process-wide registry with one background compile thread (joined at exit).
struct Registry {
    std::mutex mu;
    std::condition_variable cv;
    std::map<Key, Entry> entries;
    std::deque<JitKey> queue;
    std::thread worker;
    bool stop = false;

    ~Registry() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
            queue.clear();
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
    }
    void finish(const JitKey& k, bool ok, std::vector<char>&& cubin, std::string&& log) {
        Entry& e = entries[key_of(k)];
        e.state = ok ? State::Compiled : State::Failed;
        e.cubin = std::move(cubin);
        e.log = std::move(log);
    }
    void run() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || !queue.empty(); });
            if (stop) return;
            const JitKey k = queue.front();
            queue.pop_front();
            lk.unlock();
            std::vector<char> cubin;
            std::string log;
            const bool ok = compile_cubin(k, &cubin, &log);
            lk.lock();
            finish(k, ok, std::move(cubin), std::move(log));
            cv.notify_all();
        }
    }
    // Compiles k in the calling thread unless another thread is already doing it; returns with
    // the entry compiled, loaded or failed. Called with lk held.
    void compile_now(std::unique_lock<std::mutex>& lk, const JitKey& k) {
        Entry& e = entries[key_of(k)];
        if (e.state == State::None) {
            e.state = State::Queued;
            lk.unlock();
            std::vector<char> cubin;
            std::string log;
            const bool ok = compile_cubin(k, &cubin, &log);
            lk.lock();
            finish(k, ok, std::move(cubin), std::move(log));
            cv.notify_all();
        }
        cv.wait(lk, [&] { return entries[key_of(k)].state != State::Queued; });
    }
};

Registry& registry() {
    static Registry r;
    return r;
}

// NVRTC sets up static state of its own (and loads its builtins library) during its first
// compile, and registers exit-time teardown for it then. A compile still running in the worker
// when that teardown runs crashes the process. So before the worker starts, the calling thread
// loads NVRTC and compiles an empty kernel, and only then registers join_worker_at_exit: exit
// handlers run in reverse order of registration, so the worker is joined before NVRTC's state
// is torn down.
void prime_nvrtc() {
    Nvrtc& n = nvrtc();
    if (!n.ok) return;
    nvrtcProgram prog = nullptr;
    if (n.create(&prog, "extern \"C\" __global__ void cave_prime() {}", "cave_prime.cu", 0, nullptr, nullptr) !=
        NVRTC_SUCCESS)
        return;
    const char* opts[] = {"--gpu-architecture=sm_100a"};
    n.compile(prog, 1, opts);
    n.destroy(&prog);
}

void join_worker_at_exit() {
    Registry& R = registry();
    {
        std::lock_guard<std::mutex> g(R.mu);
        R.stop = true;
        R.queue.clear();
    }
    R.cv.notify_all();
    if (R.worker.joinable()) R.worker.join();
}

// Queues k for the background compile (starting the worker on first use). Called with R.mu held.
void queue_compile(Registry& R, const JitKey& k) {
    Entry& e = R.entries[key_of(k)];
    if (e.state != State::None || R.stop) return;
    e.state = State::Queued;
    R.queue.push_back(k);
    if (!R.worker.joinable()) {
        prime_nvrtc();
        std::atexit(join_worker_at_exit);
        R.worker = std::thread([&R] { R.run(); });
    }
    R.cv.notify_all();
}

std::atomic<uint32_t> g_loaded{0};
std::atomic<uint64_t> g_launches{0};

}  // namespace

Tick2Geometry tick2_geometry() {
    static const Tick2Geometry g = [] {
        Tick2Geometry t{(uint32_t)kJit2RowsPerThread, (uint32_t)kJit2MaxThreads, (uint32_t)kJit2CtasPerSm};
        if (const char* v = std::getenv("CAVE_TICK2_CTAS")) {
            const int c = std::atoi(v);
            if (c >= 1 && c <= 4) t.ctas_per_sm = (uint32_t)c;
        }
        if (const char* v = std::getenv("CAVE_TICK2_ROWS")) {
            const int r = std::atoi(v);
            if (r >= 1 && r <= 3) t.rows_per_thread = (uint32_t)r;
        }
        if (const char* v = std::getenv("CAVE_TICK2_THREADS")) {
            const int n = std::atoi(v);
            if (n >= 32 && n <= 1024 && n % 32 == 0) t.max_threads = (uint32_t)n;
        }
        return t;
    }();
    return g;
}

JitMode jit_mode() {
    const char* v = std::getenv("CAVE_JIT");
    if (!v || !*v || !std::strcmp(v, "async")) return JitMode::Async;
    if (!std::strcmp(v, "0") || !std::strcmp(v, "off")) return JitMode::Off;
    if (!std::strcmp(v, "1") || !std::strcmp(v, "sync")) return JitMode::Sync;
    return JitMode::Async;
}

JitKernels jit_stream_kernel(const JitKey& k, JitMode mode, bool start) {
    if (mode == JitMode::Off) return JitKernels{};
    Registry& R = registry();
    std::unique_lock<std::mutex> lk(R.mu);
    Entry* e = &R.entries[key_of(k)];
    if (e->state == State::Loaded) return e->kern;
    if (e->state == State::Failed) return JitKernels{};
    if (mode == JitMode::Sync) {
        R.compile_now(lk, k);
        e = &R.entries[key_of(k)];
    } else if (e->state == State::None) {
        if (start) queue_compile(R, k);
        return JitKernels{};
    }
    if (e->state != State::Compiled) return JitKernels{};
    cudaError_t err = cudaLibraryLoadData(&e->lib, e->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    for (int d = 0; d < 2 && err == cudaSuccess; d++) {
        err = cudaLibraryGetKernel(&e->kern.counting[d], e->lib, kJitCounting[d]);
        if (err == cudaSuccess) err = cudaLibraryGetKernel(&e->kern.derived[d], e->lib, kJitDerived[d]);
        if (err == cudaSuccess) err = cudaLibraryGetKernel(&e->kern.pair_first[d], e->lib, kJitPairFirst[d]);
        if (err == cudaSuccess) err = cudaLibraryGetKernel(&e->kern.pair[d], e->lib, kJitPair[d]);
    }
    if (err != cudaSuccess) {
        (void)cudaGetLastError();
        e->state = State::Failed;
        e->kern = JitKernels{};
        e->log = std::string("loading the specialised kernel: ") + cudaGetErrorString(err);
        return JitKernels{};
    }
    e->cubin.clear();
    e->cubin.shrink_to_fit();
    e->state = State::Loaded;
    g_loaded.fetch_add(1, std::memory_order_relaxed);
    return e->kern;
}

void jit_compile_async(const JitKey& k) {
    Registry& R = registry();
    std::lock_guard<std::mutex> lk(R.mu);
    queue_compile(R, k);
}

bool jit_compile(const JitKey& k, std::string* log) {
    Registry& R = registry();
    std::unique_lock<std::mutex> lk(R.mu);
    R.compile_now(lk, k);
    const Entry& e = R.entries[key_of(k)];
    if (log) *log = e.log;
    return e.state == State::Compiled || e.state == State::Loaded;
}

void jit_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void jit_counts(uint32_t* loaded, uint64_t* launches) {
    if (loaded) *loaded = g_loaded.load(std::memory_order_relaxed);
    if (launches) *launches = g_launches.load(std::memory_order_relaxed);
}

}  // namespace cave

extern "C" void cave_jit_stats(uint32_t* loaded, uint64_t* launches) { cave::jit_counts(loaded, launches); }
