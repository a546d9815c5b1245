// Per-device memo of launch set-up results.
//
// cudaFuncSetAttribute (the dynamic shared-memory limit of a kernel) and the
// occupancy it gives are properties of one device: a process that drives two
// GPUs must set the attribute on each of them.  PerDeviceMemo keys a cached
// integer by (kernel, device) and runs the set-up once per key under a mutex,
// so concurrent host threads and several devices are both safe.  A tag (the
// shared-memory size, say) is part of the key.  Plain C++ (no
// CUDA types), so the host-side logic is unit-tested without a GPU.
#pragma once

#include <map>
#include <mutex>
#include <tuple>

namespace mdp {

class PerDeviceMemo {
public:
    // Returns 0 and the cached value for (key, tag, dev); on the first request
    // of that triple runs setup(&value), which returns 0 on success.  A failed
    // set-up caches nothing, so the next request retries it.
    template <class Setup>
    int get(const void *key, long tag, int dev, Setup &&setup, int *value)
    {
        std::lock_guard<std::mutex> lk(mu_);
        const auto k = std::make_tuple(key, tag, dev);
        auto it = vals_.find(k);
        if (it != vals_.end()) {
            *value = it->second;
            return 0;
        }
        int v = 0;
        if (setup(&v)) return -1;
        vals_.emplace(k, v);
        *value = v;
        return 0;
    }

    size_t size()
    {
        std::lock_guard<std::mutex> lk(mu_);
        return vals_.size();
    }

private:
    std::mutex mu_;
    std::map<std::tuple<const void *, long, int>, int> vals_;
};

}  // namespace mdp
