// Internal helpers shared by the engine's translation units: the status-carrying
// exception, CUDA error checks and a device buffer owner. Nothing here is part of
// the public C ABI (include/uha_b200.h).
#pragma once

#include "uha_b200.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>

namespace uha {

// An error that carries the C-ABI status it maps to.
struct Error : std::runtime_error {
    uha_status status;
    Error(uha_status s, const std::string& message)
        : std::runtime_error(message), status(s)
    {
    }
};

[[noreturn]] inline void fail(uha_status s, const std::string& message)
{
    throw Error(s, message);
}

inline void check_cuda(cudaError_t result, const char* what)
{
    if (result != cudaSuccess) {
        fail(UHA_RUNTIME_ERROR,
             std::string(what) + ": " + cudaGetErrorString(result));
    }
}

inline uint64_t checked_mul(uint64_t a, uint64_t b, const char* what)
{
    if (b != 0 && a > std::numeric_limits<uint64_t>::max() / b) {
        fail(UHA_LENGTH_ERROR, std::string(what) + " size overflows");
    }
    return a * b;
}

inline uint64_t checked_add(uint64_t a, uint64_t b, const char* what)
{
    if (a > std::numeric_limits<uint64_t>::max() - b) {
        fail(UHA_LENGTH_ERROR, std::string(what) + " size overflows");
    }
    return a + b;
}

inline uint64_t round_up(uint64_t value, uint64_t multiple)
{
    return (value + multiple - 1) / multiple * multiple;
}

// Owner of one device allocation on the device that was current when it was
// allocated.
template <typename T>
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(uint64_t count) { allocate(count); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& other) noexcept
        : ptr_(std::exchange(other.ptr_, nullptr)),
          count_(std::exchange(other.count_, 0))
    {
    }
    DeviceBuffer& operator=(DeviceBuffer&& other) noexcept
    {
        if (this != &other) {
            release();
            ptr_ = std::exchange(other.ptr_, nullptr);
            count_ = std::exchange(other.count_, 0);
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }

    void allocate(uint64_t count)
    {
        release();
        if (count == 0) {
            return;
        }
        const uint64_t bytes = checked_mul(count, sizeof(T), "device buffer");
        void* p = nullptr;
        check_cuda(cudaMalloc(&p, bytes), "cannot allocate device memory");
        ptr_ = static_cast<T*>(p);
        count_ = count;
    }
    void release() noexcept
    {
        if (ptr_ != nullptr) {
            cudaFree(ptr_);
            ptr_ = nullptr;
            count_ = 0;
        }
    }
    T* get() const noexcept { return ptr_; }
    uint64_t size() const noexcept { return count_; }
    uint64_t bytes() const noexcept { return count_ * sizeof(T); }

private:
    T* ptr_ = nullptr;
    uint64_t count_ = 0;
};

// Owner of one pinned host allocation.
template <typename T>
class PinnedBuffer {
public:
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { release(); }
    void allocate(uint64_t count)
    {
        release();
        if (count == 0) {
            return;
        }
        void* p = nullptr;
        check_cuda(cudaMallocHost(&p, checked_mul(count, sizeof(T), "pinned")),
                   "cannot allocate pinned host memory");
        ptr_ = static_cast<T*>(p);
        count_ = count;
    }
    void release() noexcept
    {
        if (ptr_ != nullptr) {
            cudaFreeHost(ptr_);
            ptr_ = nullptr;
            count_ = 0;
        }
    }
    T* get() const noexcept { return ptr_; }
    uint64_t size() const noexcept { return count_; }

private:
    T* ptr_ = nullptr;
    uint64_t count_ = 0;
};

// Makes `device` current for the lifetime of the guard and restores the
// previous device afterwards.
class DeviceGuard {
public:
    explicit DeviceGuard(int device)
    {
        check_cuda(cudaGetDevice(&previous_), "cannot query current device");
        if (previous_ != device) {
            check_cuda(cudaSetDevice(device), "cannot select CUDA device");
        }
        changed_ = previous_ != device;
    }
    ~DeviceGuard()
    {
        if (changed_) {
            cudaSetDevice(previous_);
        }
    }
    DeviceGuard(const DeviceGuard&) = delete;
    DeviceGuard& operator=(const DeviceGuard&) = delete;

private:
    int previous_ = 0;
    bool changed_ = false;
};

void set_last_error(const char* message);

// Clears a non-sticky error left in the runtime by an earlier call whose
// status was not checked (for example a destructor), so the checks of the
// next call report only their own failures.
inline void clear_stale_cuda_error()
{
    static_cast<void>(cudaGetLastError());
}

// Runs the body of a C-ABI entry point and turns exceptions into status codes.
template <typename F>
uha_status guarded(F&& body)
{
    try {
        body();
        set_last_error("");
        return UHA_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc& e) {
        set_last_error(e.what());
        return UHA_LENGTH_ERROR;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UHA_RUNTIME_ERROR;
    }
}

constexpr int kMaxDevices = 64;

inline int current_device()
{
    int device = 0;
    check_cuda(cudaGetDevice(&device), "cannot query current device");
    if (device < 0 || device >= kMaxDevices) {
        fail(UHA_RUNTIME_ERROR, "device ordinal out of supported range");
    }
    return device;
}

}  // namespace uha
