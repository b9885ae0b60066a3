// Helpers shared by the C-ABI translation units: error recording, the
// CUDA-call and status macros, and the device scope every entry point opens.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>

#include "tdv_internal.hpp"

namespace tdv_abi {

constexpr int kMaxSide = 16384;

// Records a formatted message in the context and returns `s`.
inline tdv_status fail(tdv_ctx* ctx, tdv_status s, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return s;
}

// Makes ctx->device current for the duration of a call and restores the
// caller's device afterwards.
struct DeviceScope {
    int prev = -1;
    bool changed = false;
    cudaError_t err = cudaSuccess;
    explicit DeviceScope(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess && prev != dev) {
            err = cudaSetDevice(dev);
            changed = err == cudaSuccess;
        }
    }
    ~DeviceScope() {
        if (changed) cudaSetDevice(prev);
    }
};

// Scratch buffers grow on demand; growing waits for the device first because
// work already queued may still read the old buffer.
inline tdv_status ensure(tdv_ctx* ctx, tdv_ctx::Buf& b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return TDV_OK;
    if (b.ptr) {
        cudaDeviceSynchronize();
        if (ctx->release) ctx->release(b.ptr, ctx->alloc_user);
        else cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
    }
    void* p = nullptr;
    if (ctx->alloc) {
        p = ctx->alloc(bytes, ctx->alloc_user);
    } else if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
    }
    if (!p) return fail(ctx, TDV_ERR_OOM, "allocating %zu bytes of scratch failed", bytes);
    b.ptr = p;
    b.bytes = bytes;
    return TDV_OK;
}

}  // namespace tdv_abi

#define TDV_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return tdv_abi::fail(ctx, TDV_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define TDV_TRY(expr)                \
    do {                             \
        tdv_status s_ = (expr);      \
        if (s_ != TDV_OK) return s_; \
    } while (0)

#define TDV_DEVICE_SCOPE(ctx)                                                                   \
    tdv_abi::DeviceScope dscope_((ctx)->device);                                                \
    if (dscope_.err != cudaSuccess)                                                             \
        return tdv_abi::fail(ctx, TDV_ERR_CUDA, "selecting device %d: %s", (ctx)->device,       \
                             cudaGetErrorString(dscope_.err))
