// Shared host-side helpers: status/error propagation, CUDA checks, device buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ferrix_b200.h"

namespace fx {

// FerrixError (src/solver/error.rs:12-72) as a C++ exception carrying an fx_status
// and the variant's payload: the deck line of ParseError / UnsupportedKeyword,
// the id of NodeNotFound / ElementNotFound, and the string field (message,
// keyword, material / set / solver name, path). `text` empty = the display
// message without its variant prefix.
struct Error : std::runtime_error {
    int status;
    int64_t line = -1, id = -1;
    std::string text;
    Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
    Error(int s, const std::string& msg, int64_t line_, int64_t id_, std::string text_)
        : std::runtime_error(msg), status(s), line(line_), id(id_), text(std::move(text_)) {}
};

[[noreturn]] inline void fail(int status, const std::string& msg) { throw Error(status, msg); }
[[noreturn]] inline void fail_detail(int status, const std::string& msg, int64_t line, int64_t id,
                                     const std::string& text) {
    throw Error(status, msg, line, id, text);
}

// The last failure an entry point reported, with its payload (fx_last_error_detail).
struct ErrorRecord {
    int status = FX_OK;
    int64_t line = -1, id = -1;
    std::string text, message;
    void set(const Error& e);
    void set(int status, const std::string& message);
};

#define FX_CUDA_CHECK(expr)                                                                          \
    do {                                                                                             \
        cudaError_t _e = (expr);                                                                     \
        if (_e != cudaSuccess)                                                                       \
            ::fx::fail(FX_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e) + " @" __FILE__ ":" + \
                                    std::to_string(__LINE__));                                       \
    } while (0)

// Host wait with a deadline: polls the stream instead of blocking forever.
void stream_wait(cudaStream_t s, const char* what, double timeout_s = 120.0);
// FX_DEBUG_SYNC=1: wait for every kernel right after its launch and name it.
bool debug_sync();

// Launch bookkeeping: every kernel launch goes through FX_LAUNCH so the
// context can report how many of its own kernels ran.
extern thread_local int64_t* g_launch_counter;
#define FX_LAUNCH(kernel, grid, block, smem, stream, ...)                                            \
    do {                                                                                             \
        kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);                                  \
        if (::fx::g_launch_counter) ++*::fx::g_launch_counter;                                       \
        FX_CUDA_CHECK(cudaGetLastError());                                                           \
        if (::fx::debug_sync()) ::fx::stream_wait((stream), #kernel, 20.0);                          \
    } while (0)

// Stream-ordered device buffer (cudaMallocAsync / cudaFreeAsync).
template <typename T>
struct DBuf {
    T* ptr = nullptr;
    size_t n = 0;
    cudaStream_t stream = nullptr;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept { swap(o); }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            swap(o);
        }
        return *this;
    }
    ~DBuf() { release(); }
    void swap(DBuf& o) noexcept {
        std::swap(ptr, o.ptr);
        std::swap(n, o.n);
        std::swap(stream, o.stream);
    }
    void alloc(size_t count, cudaStream_t s) {
        if (count == n && ptr) return;
        release();
        stream = s;
        n = count;
        if (count) FX_CUDA_CHECK(cudaMallocAsync((void**)&ptr, count * sizeof(T), s));
    }
    void release() noexcept {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        n = 0;
    }
    void zero(cudaStream_t s) {
        if (n) FX_CUDA_CHECK(cudaMemsetAsync(ptr, 0, n * sizeof(T), s));
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(count, s);
        if (count) FX_CUDA_CHECK(cudaMemcpyAsync(ptr, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
    void download(T* h, size_t count, cudaStream_t s) const {
        if (count) FX_CUDA_CHECK(cudaMemcpyAsync(h, ptr, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Timer on CUDA events of one stream.
struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    EventTimer() {
        FX_CUDA_CHECK(cudaEventCreate(&a));
        FX_CUDA_CHECK(cudaEventCreate(&b));
    }
    ~EventTimer() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    void start(cudaStream_t s) { FX_CUDA_CHECK(cudaEventRecord(a, s)); }
    double stop_ms(cudaStream_t s) {
        FX_CUDA_CHECK(cudaEventRecord(b, s));
        FX_CUDA_CHECK(cudaEventSynchronize(b));
        float ms = 0.f;
        FX_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
        return ms;
    }
};

}  // namespace fx
