// TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Host shim that lets the reference's CUDA C++ sources (QC-STORM
// "bfgsMLE_dll") compile with g++ and run unmodified on the CPU, so that the
// reference itself can be executed in a container without a GPU and used to
// pin the CPU oracle.  It provides:
//   * the CUDA C++ qualifiers as no-ops (__shared__ becomes a per-OS-thread
//     static, shared by the emulated threads of one block);
//   * threadIdx / blockIdx / blockDim / gridDim and __syncthreads(), driven by
//     a coroutine SIMT block emulator (simt_emu.cpp);
//   * the fast-math intrinsics __expf / __logf mapped to libm expf / logf
//     (the only intended numerical difference from the GPU build);
//   * CUDA's min/max/abs overload semantics (fminf/fmaxf for float);
//   * the runtime API subset the reference calls, backed by host memory.
// A kernel launch `k<<<g, b, s, st>>>(args)` is rewritten by the build recipe
// (oracle/build_ref.py) into `qcs_emu_cfg(g, b, s, st).run((k), args)`.
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <algorithm>
#include <tuple>
#include <utility>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __shared__ static thread_local
#define __constant__ static
#ifndef __declspec
#define __declspec(x)
#endif

struct uint3 { unsigned int x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

void __syncthreads();

// ---- device math -----------------------------------------------------------
inline float __expf(float x) { return expf(x); }
inline float __logf(float x) { return logf(x); }
inline float __fdividef(float a, float b) { return a / b; }
inline float __powf(float a, float b) { return powf(a, b); }

inline float min(float a, float b) { return fminf(a, b); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline double min(double a, double b) { return fmin(a, b); }
inline double max(double a, double b) { return fmax(a, b); }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
inline long long min(long long a, long long b) { return a < b ? a : b; }
inline long long max(long long a, long long b) { return a > b ? a : b; }
inline unsigned short min(unsigned short a, unsigned short b) { return a < b ? a : b; }
inline unsigned short max(unsigned short a, unsigned short b) { return a > b ? a : b; }
using std::abs;
using std::isnan;

// ---- atomics (blocks run one at a time on one OS thread; relaxed is enough)
inline int atomicAdd(int *p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline unsigned int atomicAdd(unsigned int *p, unsigned int v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline float atomicAdd(float *p, float v) { float o = *p; *p = o + v; return o; }
inline int atomicMax(int *p, int v) { int o = *p; if (v > o) *p = v; return o; }

// ---- runtime API subset ----------------------------------------------------
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
typedef struct qcs_emu_stream *cudaStream_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3, cudaMemcpyDefault = 4
};
#define cudaStreamNonBlocking 1
struct cudaDeviceProp { char name[256]; int multiProcessorCount; int major; int minor; };

inline cudaError_t cudaMalloc(void **p, size_t n) { *p = calloc(n ? n : 1, 1); return *p ? cudaSuccess : cudaErrorMemoryAllocation; }
inline cudaError_t cudaMallocHost(void **p, size_t n) { return cudaMalloc(p, n); }
inline cudaError_t cudaFree(void *p) { free(p); return cudaSuccess; }
inline cudaError_t cudaFreeHost(void *p) { free(p); return cudaSuccess; }
inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { if (n) memmove(d, s, n); return cudaSuccess; }
inline cudaError_t cudaMemcpyAsync(void *d, const void *s, size_t n, cudaMemcpyKind k, cudaStream_t = nullptr) { return cudaMemcpy(d, s, n, k); }
inline cudaError_t cudaMemset(void *d, int v, size_t n) { memset(d, v, n); return cudaSuccess; }
inline cudaError_t cudaMemsetAsync(void *d, int v, size_t n, cudaStream_t = nullptr) { return cudaMemset(d, v, n); }
inline cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaStreamQuery(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
inline cudaError_t cudaStreamCreate(cudaStream_t *s) { *s = nullptr; return cudaSuccess; }
inline cudaError_t cudaStreamCreateWithPriority(cudaStream_t *s, unsigned int, int) { *s = nullptr; return cudaSuccess; }
inline cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
inline cudaError_t cudaGetLastError() { return cudaSuccess; }
inline const char *cudaGetErrorString(cudaError_t) { return "host-emulated"; }
inline cudaError_t cudaGetDeviceCount(int *c) { *c = 1; return cudaSuccess; }
inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }
inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int) {
    memset(p, 0, sizeof(*p)); strcpy(p->name, "host-emulated"); p->multiProcessorCount = 1; return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyToSymbolAsync(T &sym, const void *src, size_t n, size_t off = 0,
                                           cudaMemcpyKind = cudaMemcpyHostToDevice, cudaStream_t = nullptr) {
    memcpy(reinterpret_cast<char *>(&sym) + off, src, n);
    return cudaSuccess;
}
template <class T>
inline cudaError_t cudaMemcpyToSymbol(T &sym, const void *src, size_t n, size_t off = 0,
                                      cudaMemcpyKind = cudaMemcpyHostToDevice) {
    memcpy(reinterpret_cast<char *>(&sym) + off, src, n);
    return cudaSuccess;
}

// ---- kernel launch emulation -----------------------------------------------
// Runs every block of the grid in order; inside a block the threads are
// coroutines that switch at __syncthreads() (see simt_emu.cpp).
typedef void (*qcs_emu_thread_fn)(void *ctx);
void qcs_emu_run_block(unsigned int nthreads, qcs_emu_thread_fn fn, void *ctx);

struct qcs_emu_cfg {
    dim3 grid, block;
    qcs_emu_cfg(dim3 g, dim3 b, size_t = 0, cudaStream_t = nullptr) : grid(g), block(b) {}

    template <class... P, class... A>
    void run(void (*k)(P...), A &&...args) const {
        struct Ctx {
            void (*k)(P...);
            std::tuple<P...> a;
        } ctx{k, std::tuple<P...>(static_cast<P>(args)...)};
        gridDim = grid;
        blockDim = block;
        const unsigned int nb = grid.x * grid.y * grid.z;
        const unsigned int nt = block.x * block.y * block.z;
        for (unsigned int b = 0; b < nb; ++b) {
            blockIdx.x = b % grid.x;
            blockIdx.y = (b / grid.x) % grid.y;
            blockIdx.z = b / (grid.x * grid.y);
            qcs_emu_run_block(nt, [](void *c) {
                Ctx *x = static_cast<Ctx *>(c);
                std::tuple<P...> copy = x->a;  // kernels may modify by-value parameters
                std::apply(x->k, copy);
            }, &ctx);
        }
    }
};
