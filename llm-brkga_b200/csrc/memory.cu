// memory.cu -- device memory for problems and engines: a stream-ordered pool per device,
// owned by the library.  Freed blocks stay cached in the pool (release threshold = max),
// so creating and destroying engines at serving rates costs no device-wide
// synchronisation and no page mapping after the first time.
#include <cstdint>
#include <map>
#include <mutex>

#include "engine.h"

namespace bk {

static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static cudaError_t pool_of(int dev, cudaMemPool_t* out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    g_pools[dev] = pool;
    *out = pool;
    return cudaSuccess;
}

int32_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    cudaMemPool_t pool;
    if (e == cudaSuccess) e = pool_of(dev, &pool);
    if (e != cudaSuccess) return cuda_fail(e, "memory pool");
    e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(BRKGA_ERR_OOM, std::string("device allocation of ") + std::to_string(bytes) + " bytes: " +
                                       cudaGetErrorString(e));
    }
    return BRKGA_OK;
}

void dev_free(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}

// bytes the pool holds but has not handed out (reusable without a new device allocation)
size_t pool_spare(int dev) {
    cudaMemPool_t pool;
    if (pool_of(dev, &pool) != cudaSuccess) return 0;
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    return reserved > used ? (size_t)(reserved - used) : 0;
}

size_t pool_reserved(int dev) {
    cudaMemPool_t pool;
    if (pool_of(dev, &pool) != cudaSuccess) return 0;
    uint64_t v = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &v);
    return (size_t)v;
}

}  // namespace bk
