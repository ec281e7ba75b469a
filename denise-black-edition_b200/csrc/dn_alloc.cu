// Device memory of the library: models, shots (wavefields, snapshot stores,
// checkpoints), batch descriptors and per-call buffers.  Freed blocks are
// kept per device and handed to the next request of nearly the same size
// (at most 1/8 larger), so successive shot batches reuse their multi-GB
// snapshot stores instead of freeing and mapping them again: cudaFree of an
// 18 GB FP16 store took ~18 ms, a quarter of a second per batch of seven
// 1700 x 500, NT 4000 gradient shots.  (A stream-ordered cudaMemPool with an
// unlimited release threshold reuses as well, but grew ~20x slower than
// cudaMalloc on a B200.)
//
// dn_free waits for the device before it caches a block, as cudaFree does, so
// no kernel still uses a block that is handed out again.  A request that
// cudaMalloc cannot serve releases the cached blocks of that device and tries
// once more; dn_device_memory counts cached bytes as free, and dn_device_trim
// releases them for allocators outside the library.  DN_POOL=0 in the
// environment makes dn_malloc / dn_free plain cudaMalloc / cudaFree.
#include <cuda_runtime.h>

#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>

#include "denise_b200.h"
#include "dn_internal.h"

namespace {

struct Block {
    size_t bytes;
    int device;
};

std::mutex g_mu;
std::unordered_map<void *, Block> g_live;               // handed out
std::map<int, std::multimap<size_t, void *>> g_cached;   // device -> size -> freed block
std::map<int, size_t> g_cached_bytes;

bool pool_enabled()
{
    static const bool on = [] {
        const char *e = getenv("DN_POOL");
        return !(e && e[0] == '0');
    }();
    return on;
}

// frees every cached block of `device` (the current device); caller holds g_mu
void release_cached(int device)
{
    auto &c = g_cached[device];
    for (auto &kv : c) cudaFree(kv.second);
    c.clear();
    g_cached_bytes[device] = 0;
}

}   // namespace

cudaError_t dn_malloc_bytes(void **p, size_t bytes)
{
    *p = nullptr;
    if (!pool_enabled()) return cudaMalloc(p, bytes);
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(g_mu);
    auto &c = g_cached[device];
    auto it = c.lower_bound(bytes);
    if (it != c.end() && it->first - bytes <= bytes / 8) {
        *p = it->second;
        g_live[*p] = {it->first, device};
        g_cached_bytes[device] -= it->first;
        c.erase(it);
        return cudaSuccess;
    }
    e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation && !c.empty()) {
        cudaGetLastError();
        release_cached(device);
        e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    g_live[*p] = {bytes, device};
    return e;
}

void dn_free(void *p)
{
    if (!p) return;
    if (!pool_enabled()) {
        cudaFree(p);
        return;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_live.find(p);
    if (it == g_live.end()) {   // not from dn_malloc
        cudaFree(p);
        return;
    }
    const Block b = it->second;
    g_live.erase(it);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b.device) cudaSetDevice(b.device);
    cudaDeviceSynchronize();   // as cudaFree: nothing still running may use p when it is handed out again
    if (cur != b.device) cudaSetDevice(cur);
    g_cached[b.device].emplace(b.bytes, p);
    g_cached_bytes[b.device] += b.bytes;
}

size_t dn_pool_idle_bytes(int device)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_cached_bytes.find(device);
    return it == g_cached_bytes.end() ? 0 : it->second;
}

extern "C" int dn_device_trim(int device)
{
    std::lock_guard<std::mutex> lk(g_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) release_cached(device);
    cudaSetDevice(cur);
    if (e != cudaSuccess) return dn_fail(DN_EDEVICE, "dn_device_trim(%d): %s", device, cudaGetErrorString(e));
    return DN_OK;
}
