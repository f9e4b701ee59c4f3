// Library-level entry points and state: ABI version, per-thread error
// messages, the per-device memory pool for per-call scratch.
#include "prr_internal.h"

#include <cstring>
#include <mutex>
#include <vector>

namespace prr {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    set_error(msg);
    return code;
}

// The library's stream-ordered memory pool of a device: freed blocks stay in
// it (up to a 4 GiB release threshold) for the next calls instead of going
// back to the driver at every synchronisation, as the device's default pool
// would do. Created on first use, one per device.
cudaError_t library_pool(cudaMemPool_t *out) {
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    std::lock_guard<std::mutex> g(mu);
    if ((int) pools.size() <= dev)
        pools.resize(dev + 1, nullptr);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess)
            return e;
        uint64_t keep = uint64_t(4) << 30;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    *out = pools[dev];
    return cudaSuccess;
}

} // namespace prr

extern "C" {

int prr_abi_version(void) { return PRR_ABI_VERSION; }

int prr_last_error(char *buf, size_t len) {
    const std::string &e = prr::g_last_error;
    if (buf && len > 0) {
        const size_t n = std::min(len - 1, e.size());
        std::memcpy(buf, e.data(), n);
        buf[n] = '\0';
    }
    return (int) e.size();
}

} // extern "C"
