// cmd_internal.h -- shared helpers of the C-ABI implementation (not installed).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "cmd.h"

namespace cmd {

// Records `msg` as this host thread's last error and returns `code`.
int fail(int code, const std::string& msg);
// Clears the last error (called at the start of every public entry point).
void clear_error();

// A device allocation that only grows; the owner calls release().
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n) {
        if (n <= bytes) return CMD_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, n);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(CMD_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        bytes = n;
        return CMD_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Page-locked host buffer, grown on demand (device-to-host copies into it run
// at full link speed and asynchronously).
struct HostBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t n) {
        if (n <= bytes) return CMD_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(CMD_ERR_OOM, std::string("cudaHostAlloc: ") + cudaGetErrorString(e));
        }
        bytes = n;
        return CMD_OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace cmd
