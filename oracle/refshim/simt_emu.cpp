// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Coroutine SIMT block emulator behind oracle/refshim/cuda_runtime.h.  Each
// emulated CUDA thread of a block runs on its own ucontext stack; a thread
// that reaches __syncthreads() parks, and the scheduler releases the barrier
// once every thread of the block is parked or finished.  Threads are resumed
// in threadIdx order, so a block's atomics and stores happen in a fixed,
// reproducible order.
#include <ucontext.h>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "cuda_runtime.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

namespace {

enum { kRunnable = 0, kAtBarrier = 1, kDone = 2 };
constexpr size_t kStackBytes = 256 * 1024;

struct Block {
    ucontext_t sched;
    std::vector<ucontext_t> ctx;
    std::vector<int> state;
    std::vector<char> stacks;
    qcs_emu_thread_fn fn = nullptr;
    void *arg = nullptr;
    unsigned int cur = 0;
};

thread_local Block *g_block = nullptr;

void set_thread_index(unsigned int t) {
    threadIdx.x = t % blockDim.x;
    threadIdx.y = (t / blockDim.x) % blockDim.y;
    threadIdx.z = t / (blockDim.x * blockDim.y);
}

void trampoline() {
    Block *b = g_block;
    b->fn(b->arg);
    b->state[b->cur] = kDone;
    // returning resumes uc_link (the scheduler)
}

}  // namespace

void __syncthreads() {
    Block *b = g_block;
    if (!b) return;
    const unsigned int t = b->cur;
    b->state[t] = kAtBarrier;
    swapcontext(&b->ctx[t], &b->sched);
    set_thread_index(t);
}

void qcs_emu_run_block(unsigned int nthreads, qcs_emu_thread_fn fn, void *arg) {
    thread_local Block blk;
    Block &b = blk;
    b.fn = fn;
    b.arg = arg;
    if (b.ctx.size() < nthreads) {
        b.ctx.resize(nthreads);
        b.stacks.resize(static_cast<size_t>(nthreads) * kStackBytes);
    }
    b.state.assign(nthreads, kRunnable);
    for (unsigned int t = 0; t < nthreads; ++t) {
        getcontext(&b.ctx[t]);
        b.ctx[t].uc_stack.ss_sp = b.stacks.data() + static_cast<size_t>(t) * kStackBytes;
        b.ctx[t].uc_stack.ss_size = kStackBytes;
        b.ctx[t].uc_link = &b.sched;
        makecontext(&b.ctx[t], trampoline, 0);
    }
    Block *saved = g_block;
    g_block = &b;
    for (;;) {
        for (unsigned int t = 0; t < nthreads; ++t) {
            if (b.state[t] != kRunnable) continue;
            b.cur = t;
            set_thread_index(t);
            swapcontext(&b.sched, &b.ctx[t]);
        }
        bool any_waiting = false;
        for (unsigned int t = 0; t < nthreads; ++t) {
            if (b.state[t] == kAtBarrier) { b.state[t] = kRunnable; any_waiting = true; }
        }
        if (!any_waiting) break;
    }
    g_block = saved;
}
