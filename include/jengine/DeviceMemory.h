// DeviceMemory.h -- RAII device buffer, the element type of device pipes.
//
// Behaviour of the reference's CUDA/DeviceMemory.h and DeviceMemory.cpp:19-70:
// construction allocates (an allocation failure throws an Exception whose
// message starts with "CUDA failed to malloc ", the prefix JEngine's retry
// loop matches, JEngine/JEngine.cpp:413-421), copying copies the device
// contents, moving steals the allocation.
#pragma once

#include <cstddef>

#include "Common.h"

namespace JEngine {

void* DeviceAlloc(size_t bytes);          // throws "CUDA failed to malloc ..."
void DeviceFree(void* p) noexcept;
void DeviceCopy(void* dst, const void* src, size_t bytes);       // device -> device
void CopyToDevice(void* dst, const void* src, size_t bytes);     // host -> device
void CopyToHost(void* dst, const void* src, size_t bytes);       // device -> host

template <class T>
class DeviceMemory {
public:
    explicit DeviceMemory(size_t n = 0) : n(n), p(n ? static_cast<T*>(DeviceAlloc(n * sizeof(T))) : nullptr) {}
    DeviceMemory(const DeviceMemory& o) : DeviceMemory(o.n) {
        if (n) DeviceCopy(p, o.p, n * sizeof(T));
    }
    DeviceMemory(DeviceMemory&& o) noexcept : n(o.n), p(o.p) {
        o.n = 0;
        o.p = nullptr;
    }
    DeviceMemory& operator=(const DeviceMemory& o) {
        if (this != &o) {
            DeviceMemory t(o);
            swap(t);
        }
        return *this;
    }
    DeviceMemory& operator=(DeviceMemory&& o) noexcept {
        swap(o);
        return *this;
    }
    ~DeviceMemory() { DeviceFree(p); }

    void swap(DeviceMemory& o) noexcept {
        std::swap(n, o.n);
        std::swap(p, o.p);
    }
    T* Data() { return p; }
    const T* Data() const { return p; }
    const T* CData() const { return p; }
    size_t Size() const { return n; }

private:
    size_t n;
    T* p;
};

}  // namespace JEngine
