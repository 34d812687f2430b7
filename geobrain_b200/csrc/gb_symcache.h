// Cache of a device symbol's address per (device, CUDA context).
//
// The address of a file-scope __device__ array belongs to the module the
// driver loaded into one context.  After cudaDeviceReset, or in a host that
// runs its own driver-API contexts on the device, the module is loaded again
// and the array may sit elsewhere: an address cached by device alone would
// then point at memory this library no longer owns.  Entries are therefore
// keyed by the device ordinal and the context's unique ID (cuCtxGetId, never
// reused within a process); a call on a context not seen before looks the
// address up afresh.  Pure C++, so that it can be checked without a GPU.
#pragma once

#include <cstddef>
#include <mutex>

namespace gb {
namespace host {

template <int N>
class SymbolAddressCache {
public:
    // The address for (dev, ctx_id): the cached one, or lookup(&addr) (which
    // returns 0 on success) for a new key.  A full table drops its oldest
    // entry.  Returns what lookup returned on a failed lookup, else 0.
    template <class Lookup>
    int get(int dev, unsigned long long ctx_id, Lookup lookup, void **out)
    {
        std::lock_guard<std::mutex> lock(mu_);
        for (int i = 0; i < n_; ++i)
            if (e_[i].dev == dev && e_[i].ctx == ctx_id) {
                *out = e_[i].addr;
                return 0;
            }
        void *addr = nullptr;
        if (int rc = lookup(&addr)) return rc;
        ++lookups_;
        if (n_ == N) {
            for (int i = 1; i < N; ++i) e_[i - 1] = e_[i];
            --n_;
        }
        e_[n_++] = Entry{dev, ctx_id, addr};
        *out = addr;
        return 0;
    }
    // Lookups made so far (misses that succeeded).
    long long lookups() const { return lookups_; }

private:
    struct Entry {
        int dev;
        unsigned long long ctx;
        void *addr;
    };
    std::mutex mu_;
    Entry e_[N] = {};
    int n_ = 0;
    long long lookups_ = 0;
};

}  // namespace host
}  // namespace gb
