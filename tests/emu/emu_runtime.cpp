// CPU emulation of the CUDA execution model -- TEST INFRASTRUCTURE ONLY (see cuda_runtime.h).
//
// A launch runs its blocks one after the other; the threads of a block are fibers (ucontext)
// that run until they finish or reach a barrier.  __syncthreads releases the block's fibers
// when every live thread has arrived; __syncwarp and the warp shuffles release the lanes of a
// warp named in the mask once they have all arrived, and a shuffle then reads its partner's
// value from the generation it arrived in.  A block whose live fibers all wait at barriers that
// can no longer be released is a deadlock: reported and the process aborts.  Streams execute
// their work at once (every call is in stream order and synchronous), except while a stream
// is being captured, when launches, copies and sets are recorded for graph replay.
#include <sys/mman.h>
#include <ucontext.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <vector>

#include "cuda_runtime.h"

uint3 threadIdx, blockIdx;
dim3 blockDim, gridDim;

namespace {

cudaError_t g_last = cudaSuccess;

struct Stream {
    bool capturing = false;
    std::vector<std::function<void()>> ops;
};
Stream g_default;
Stream* stream_of(cudaStream_t st) { return st ? (Stream*)st : &g_default; }

struct Graph {
    std::vector<std::function<void()>> ops;
};

struct Event {
    double t = 0.0;
};

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Either run `op` now or, while `st` is being captured, append it to the capture.
void enqueue(cudaStream_t st, std::function<void()> op) {
    Stream* s = stream_of(st);
    if (s->capturing) s->ops.push_back(std::move(op));
    else op();
}

std::map<const void*, int> g_max_dyn;   // kernel -> cudaFuncAttributeMaxDynamicSharedMemorySize

// ---------------------------------------------------------------- fibers
enum { READY = 0, WAIT_BLOCK = 1, WAIT_WARP = 2, DONE = 3 };
const size_t STACK = 512 * 1024;

struct Fiber {
    ucontext_t ctx;
    int state;
    uint3 tid;
    int lane, warp;
};
struct Warp {
    unsigned arrived, gen, mask;
    uint64_t val[2][32];
};

std::vector<Fiber> g_fib;
std::vector<char*> g_stacks;
std::vector<Warp> g_warps;
ucontext_t g_sched;
int g_cur = -1, g_n = 0, g_done = 0, g_bar = 0;
bool g_in_kernel = false;
const std::function<void()>* g_body = nullptr;
std::vector<unsigned char> g_dyn;

// HSBEMU_ORDER=reverse: blocks run last to first and the threads of a block are resumed from
// the highest index down; HSBEMU_ORDER=shuffle: both in a random order (HSBEMU_SEED), drawn
// anew for every launch and every pass over a block's threads.  A kernel that depends on an
// order the GPU does not promise (a missing barrier, a block reading another block's output)
// then gives different results.
enum { ORDER_FORWARD = 0, ORDER_REVERSE = 1, ORDER_SHUFFLE = 2 };
int schedule_order() {
    static const int o = [] {
        const char* s = getenv("HSBEMU_ORDER");
        if (s && strcmp(s, "reverse") == 0) return (int)ORDER_REVERSE;
        if (s && strcmp(s, "shuffle") == 0) return (int)ORDER_SHUFFLE;
        return (int)ORDER_FORWARD;
    }();
    return o;
}
bool reverse_order() { return schedule_order() == ORDER_REVERSE; }

uint64_t next_random() {      // xorshift64*
    static uint64_t x = [] {
        const char* s = getenv("HSBEMU_SEED");
        const uint64_t v = s ? strtoull(s, nullptr, 10) : 1;
        return v ? v : 1;
    }();
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return x * 0x2545F4914F6CDD1DULL;
}

void shuffle(std::vector<int>& v) {
    for (size_t i = v.size(); i > 1; i--) std::swap(v[i - 1], v[next_random() % i]);
}

char* stack_at(int i) {
    while ((int)g_stacks.size() <= i) {
        void* p = mmap(nullptr, STACK + 4096, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
        if (p == MAP_FAILED) {
            fprintf(stderr, "hsbemu: out of memory for fiber stacks\n");
            abort();
        }
        mprotect(p, 4096, PROT_NONE);   // guard page below the stack
        g_stacks.push_back((char*)p + 4096);
    }
    return g_stacks[i];
}

unsigned live_lanes(int w) {
    unsigned m = 0;
    for (int l = 0; l < 32; l++) {
        const int i = w * 32 + l;
        if (i < g_n && g_fib[i].state != DONE) m |= 1u << l;
    }
    return m;
}

void release_block() {
    for (int i = 0; i < g_n; i++)
        if (g_fib[i].state == WAIT_BLOCK) g_fib[i].state = READY;
    g_bar = 0;
}

void release_warp(int w) {
    Warp& W = g_warps[w];
    for (int l = 0; l < 32; l++) {
        const int i = w * 32 + l;
        if (i < g_n && g_fib[i].state == WAIT_WARP) g_fib[i].state = READY;
    }
    W.arrived = 0;
    W.gen++;
}

// After a fiber finishes, barriers it no longer has to reach may be complete.
void check_releases(int w) {
    if (g_bar > 0 && g_bar == g_n - g_done) release_block();
    Warp& W = g_warps[w];
    if (W.arrived) {
        const unsigned part = W.mask & live_lanes(w);
        if ((W.arrived & part) == part) release_warp(w);
    }
}

void yield_to_scheduler() {
    const int me = g_cur;
    swapcontext(&g_fib[me].ctx, &g_sched);
}

void trampoline() {
    (*g_body)();
    Fiber& f = g_fib[g_cur];
    f.state = DONE;
    g_done++;
    check_releases(f.warp);
}

void run_block(int n) {
    g_n = n;
    g_done = 0;
    g_bar = 0;
    g_fib.resize(n);
    g_warps.assign((n + 31) / 32, Warp{0, 0, 0, {}});
    const unsigned bx = blockDim.x, by = blockDim.y;
    for (int i = 0; i < n; i++) {
        Fiber& f = g_fib[i];
        f.state = READY;
        f.tid = uint3{(unsigned)(i % bx), (unsigned)((i / bx) % by), (unsigned)(i / (bx * by))};
        f.lane = i & 31;
        f.warp = i >> 5;
        getcontext(&f.ctx);
        f.ctx.uc_stack.ss_sp = stack_at(i);
        f.ctx.uc_stack.ss_size = STACK;
        f.ctx.uc_link = &g_sched;
        makecontext(&f.ctx, trampoline, 0);
    }
    const bool rev = reverse_order(), shuf = schedule_order() == ORDER_SHUFFLE;
    std::vector<int> perm(n);
    for (int j = 0; j < n; j++) perm[j] = rev ? n - 1 - j : j;
    while (g_done < n) {
        bool ran = false;
        if (shuf) shuffle(perm);
        for (int j = 0; j < n; j++) {
            const int i = perm[j];
            if (g_fib[i].state != READY) continue;
            g_cur = i;
            threadIdx = g_fib[i].tid;
            swapcontext(&g_sched, &g_fib[i].ctx);
            ran = true;
        }
        if (!ran) {
            fprintf(stderr, "hsbemu: deadlock in block (%u, %u, %u): %d of %d threads wait at barriers that cannot "
                            "complete\n", blockIdx.x, blockIdx.y, blockIdx.z, n - g_done, n);
            abort();
        }
    }
    g_cur = -1;
}

void run_grid(const hsbemu::Cfg& c, const std::function<void()>& body) {
    const int n = (int)(c.block.x * c.block.y * c.block.z);
    blockDim = c.block;
    gridDim = c.grid;
    g_body = &body;
    g_in_kernel = true;
    // exactly the launch's dynamic shared memory (an AddressSanitizer build reports any access
    // past it); uninitialised shared memory reads as NaN / all ones
    g_dyn.assign(c.smem ? c.smem : 1, 0xFF);
    const long nb = (long)c.grid.x * c.grid.y * c.grid.z;
    std::vector<int> order(nb);
    for (long b = 0; b < nb; b++) order[b] = (int)(reverse_order() ? nb - 1 - b : b);
    if (schedule_order() == ORDER_SHUFFLE) shuffle(order);
    for (long q = 0; q < nb; q++) {
        const long b = order[q];
        blockIdx = uint3{(unsigned)(b % c.grid.x), (unsigned)((b / c.grid.x) % c.grid.y),
                         (unsigned)(b / ((long)c.grid.x * c.grid.y))};
        memset(g_dyn.data(), 0xFF, g_dyn.size());
        run_block(n);
    }
    g_in_kernel = false;
    g_body = nullptr;
}

}  // namespace

// ---------------------------------------------------------------- device built-ins
void __syncthreads() {
    if (!g_in_kernel || g_cur < 0) return;
    g_bar++;
    if (g_bar == g_n - g_done) {
        // the last thread to arrive also goes back to the scheduler, so that after every
        // barrier the block's threads resume in the scheduling order (forward or reverse)
        release_block();
        yield_to_scheduler();
        return;
    }
    g_fib[g_cur].state = WAIT_BLOCK;
    yield_to_scheduler();
}

static uint64_t warp_op(unsigned mask, uint64_t v, int xor_mask, bool shuffle) {
    if (!g_in_kernel || g_cur < 0) return v;
    Fiber& f = g_fib[g_cur];
    const int w = f.warp, lane = f.lane;
    Warp& W = g_warps[w];
    const unsigned g = W.gen;
    W.val[g & 1][lane] = v;
    W.arrived |= 1u << lane;
    W.mask = mask;
    const unsigned part = mask & live_lanes(w);
    if ((W.arrived & part) == part) {
        release_warp(w);
        yield_to_scheduler();     // as at a block barrier: resume in the scheduling order
    } else {
        f.state = WAIT_WARP;
        yield_to_scheduler();
    }
    if (!shuffle) return 0;
    return g_warps[w].val[g & 1][(lane ^ xor_mask) & 31];
}

void __syncwarp(unsigned mask) { warp_op(mask, 0, 0, false); }

uint64_t hsbemu_shfl_xor(unsigned mask, uint64_t bits, int lane_mask) { return warp_op(mask, bits, lane_mask, true); }

// ---------------------------------------------------------------- launches
namespace hsbemu {

void set_attribute(const void* fn, int attr, int value) {
    if (attr == cudaFuncAttributeMaxDynamicSharedMemorySize) g_max_dyn[fn] = value;
}

void* dyn_smem() { return g_dyn.data(); }

void submit(const void* fn, const Cfg& c, std::function<void()> body) {
    const unsigned long threads = (unsigned long)c.block.x * c.block.y * c.block.z;
    if (threads == 0 || threads > 1024 || c.block.z > 64 || c.grid.x == 0 || c.grid.y == 0 || c.grid.z == 0 ||
        c.grid.y > 65535 || c.grid.z > 65535) {
        fprintf(stderr, "hsbemu: invalid launch configuration grid (%u, %u, %u) block (%u, %u, %u)\n", c.grid.x,
                c.grid.y, c.grid.z, c.block.x, c.block.y, c.block.z);
        g_last = cudaErrorInvalidConfiguration;
        return;
    }
    auto it = g_max_dyn.find(fn);
    const size_t limit = (it != g_max_dyn.end() && it->second > 48 * 1024) ? (size_t)it->second : 48 * 1024;
    if (c.smem > limit || c.smem > 227 * 1024) {
        fprintf(stderr, "hsbemu: %zu bytes of dynamic shared memory above the kernel's limit %zu\n", c.smem, limit);
        g_last = cudaErrorInvalidValue;
        return;
    }
    const Cfg cfg = c;
    enqueue(c.st, [cfg, body]() { run_grid(cfg, body); });
}

}  // namespace hsbemu

// ---------------------------------------------------------------- runtime API
cudaError_t cudaMalloc(void** p, size_t n) {
    if (!p) return cudaErrorInvalidValue;
    if (posix_memalign(p, 256, n ? n : 1) != 0) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    memset(*p, 0xA5, n);   // device memory starts with garbage
    return cudaSuccess;
}
cudaError_t cudaMallocHost(void** p, size_t n) { return cudaMalloc(p, n); }
cudaError_t cudaFree(void* p) {
    free(p);
    return cudaSuccess;
}
cudaError_t cudaFreeHost(void* p) {
    free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, cudaMemcpyKind) {
    if (stream_of(0)->capturing) return cudaErrorStreamCaptureUnsupported;
    if (n) memmove(dst, src, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t n, cudaMemcpyKind, cudaStream_t st) {
    enqueue(st, [dst, src, n]() {
        if (n) memmove(dst, src, n);
    });
    return cudaSuccess;
}
cudaError_t cudaMemset(void* p, int v, size_t n) {
    if (n) memset(p, v, n);
    return cudaSuccess;
}
cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t st) {
    enqueue(st, [p, v, n]() {
        if (n) memset(p, v, n);
    });
    return cudaSuccess;
}
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* st, unsigned) {
    *st = (cudaStream_t) new Stream();
    return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t st) {
    delete (Stream*)st;
    return cudaSuccess;
}
cudaError_t cudaStreamSynchronize(cudaStream_t st) {
    return stream_of(st)->capturing ? cudaErrorStreamCaptureUnsupported : cudaSuccess;
}
cudaError_t cudaStreamBeginCapture(cudaStream_t st, cudaStreamCaptureMode) {
    Stream* s = stream_of(st);
    if (s->capturing) return cudaErrorInvalidValue;
    s->capturing = true;
    s->ops.clear();
    return cudaSuccess;
}
cudaError_t cudaStreamEndCapture(cudaStream_t st, cudaGraph_t* g) {
    Stream* s = stream_of(st);
    if (!s->capturing) return cudaErrorInvalidValue;
    Graph* G = new Graph();
    G->ops.swap(s->ops);
    s->capturing = false;
    *g = (cudaGraph_t)G;
    return cudaSuccess;
}
cudaError_t cudaGraphInstantiate(cudaGraphExec_t* e, cudaGraph_t g, unsigned long long) {
    *e = (cudaGraphExec_t) new Graph(*(Graph*)g);
    return cudaSuccess;
}
cudaError_t cudaGraphLaunch(cudaGraphExec_t e, cudaStream_t st) {
    Graph* G = (Graph*)e;
    enqueue(st, [G]() {
        for (auto& op : G->ops) op();
    });
    return cudaSuccess;
}
cudaError_t cudaGraphDestroy(cudaGraph_t g) {
    delete (Graph*)g;
    return cudaSuccess;
}
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t e) {
    delete (Graph*)e;
    return cudaSuccess;
}
cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = (cudaEvent_t) new Event();
    return cudaSuccess;
}
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned) { return cudaEventCreate(e); }
cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete (Event*)e;
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t st) {
    Event* E = (Event*)e;
    enqueue(st, [E]() { E->t = now_ms(); });
    return cudaSuccess;
}
cudaError_t cudaEventQuery(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = (float)(((Event*)b)->t - ((Event*)a)->t);
    return cudaSuccess;
}
cudaError_t cudaGetLastError() {
    const cudaError_t e = g_last;
    g_last = cudaSuccess;
    return e;
}
const char* cudaGetErrorString(cudaError_t e) {
    switch (e) {
        case cudaSuccess: return "no error (emulated)";
        case cudaErrorInvalidValue: return "invalid argument (emulated)";
        case cudaErrorMemoryAllocation: return "out of memory (emulated)";
        case cudaErrorInvalidConfiguration: return "invalid configuration argument (emulated)";
        case cudaErrorStreamCaptureUnsupported: return "operation not permitted when stream is capturing (emulated)";
        default: return "error (emulated)";
    }
}
cudaError_t cudaGetDevice(int* dev) {
    *dev = 0;
    return cudaSuccess;
}
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int) {
    if (a == cudaDevAttrMultiProcessorCount) {
        const char* s = getenv("HSBEMU_SMS");
        *v = s ? atoi(s) : 2;
        if (*v < 1) *v = 1;
        return cudaSuccess;
    }
    return cudaErrorInvalidValue;
}
cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int) {
    memset(p, 0, sizeof(*p));
    strcpy(p->name, "CPU emulation of CUDA");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    p->totalGlobalMem = (size_t)64 << 30;
    p->sharedMemPerBlock = 48 * 1024;
    p->totalConstMem = 64 * 1024;
    p->textureAlignment = 512;
    p->regsPerBlock = 65536;
    p->warpSize = 32;
    p->maxThreadsPerBlock = 1024;
    p->maxThreadsDim[0] = p->maxThreadsDim[1] = 1024;
    p->maxThreadsDim[2] = 64;
    p->maxGridSize[0] = 2147483647;
    p->maxGridSize[1] = p->maxGridSize[2] = 65535;
    p->major = 10;
    p->clockRate = 1000000;
    p->multiProcessorCount = sms;
    return cudaSuccess;
}
cudaError_t cudaThreadSynchronize() { return cudaSuccess; }
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
