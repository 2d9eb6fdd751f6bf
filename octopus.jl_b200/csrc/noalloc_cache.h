// Per-device cache of a static device array's address for the allocation-free entry point.
//
// In host code the name of a `static __device__` array is only a host-side stand-in; kernels must be
// given the address cudaGetSymbolAddress returns with the device current.  That address belongs to the
// module loaded into the device's current context, so a cached address is valid only for the context it
// was looked up in: after cudaDeviceReset (or CUDA.jl's device_reset!) the primary context, and the module
// with it, are destroyed and a new context loads the module at a possibly different address.  Each slot
// therefore keeps the context handle beside the address and looks the address up again when the current
// context differs.  Plain C++ with no CUDA types, so the logic is testable on a machine without a GPU.
#pragma once
#include <mutex>

namespace octo {

template <int kMaxDevices>
class SymbolAddressCache {
public:
    // The address for `device` in context `ctx`: the cached one when it was looked up in the same context,
    // else resolve() (called with the device current; returns nullptr on failure, which is not cached).
    // Returns nullptr for an out-of-range device or a failed lookup.
    template <class Resolve>
    void *lookup(int device, const void *ctx, Resolve resolve) {
        if (device < 0 || device >= kMaxDevices) return nullptr;
        std::lock_guard<std::mutex> lock(mutex_);
        Slot &s = slot_[device];
        if (s.addr && s.ctx == ctx) return s.addr;
        void *a = resolve();
        if (!a) return nullptr;
        s.ctx = ctx;
        s.addr = a;
        ++lookups_;
        return a;
    }
    // Successful resolve() calls so far (a test observes re-lookups through it).
    long long lookups() const { return lookups_; }

private:
    struct Slot {
        const void *ctx = nullptr;
        void *addr = nullptr;
    };
    Slot slot_[kMaxDevices];
    std::mutex mutex_;
    long long lookups_ = 0;
};

}  // namespace octo
