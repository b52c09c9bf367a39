// Minimal runtime under the GROUP BY path: error strings, device properties, stream-ordered
// allocation and the memory helpers of the C ABI.  It stands in for the reference's Context /
// GPUMemory / CudaMemAllocator layer (qikkDB/QueryEngine/Context.cu:20-139,
// qikkDB/QueryEngine/GPUCore/GPUMemory.cuh:89-236, qikkDB/QueryEngine/CudaMemAllocator.h:11-60):
// instead of a best-fit allocator over one reserved block, device memory comes from CUDA's
// stream-ordered pool with its release threshold raised so freed blocks are reused.
#include <atomic>
#include <mutex>
#include <vector>

#include "qdb_common.cuh"

namespace qdb {

static thread_local std::string g_last_error = "";
static std::atomic<int64_t> g_launches{0};

void note_launch(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_last_error(const std::string& msg) { g_last_error = msg; }

int32_t fail(int32_t code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

int32_t cuda_fail(cudaError_t err, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(err) + " (" + cudaGetErrorString(err) + ")";
    if (err == cudaErrorMemoryAllocation) return QDB_ERR_NOMEM;
    if (err == cudaErrorNoDevice || err == cudaErrorInsufficientDriver) return QDB_NOT_FOUND;
    return QDB_ERR_CUDA;
}

const DeviceInfo& device_info() {
    static std::mutex mu;
    static std::vector<DeviceInfo> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (static_cast<int>(cache.size()) <= dev) cache.resize(dev + 1);
    DeviceInfo& di = cache[dev];
    if (di.device != dev) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
            di.sm_count = prop.multiProcessorCount;
            di.max_smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
            di.l2_bytes = prop.l2CacheSize;
        }
        // Keep freed pool blocks cached instead of returning them to the driver at every sync.
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        di.device = dev;
    }
    return di;
}

int32_t dev_alloc(void** p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    if (bytes == 0) return QDB_OK;
    device_info();
    cudaError_t e = cudaMallocAsync(p, bytes, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return cuda_fail(e, "cudaMallocAsync");
    }
    return QDB_OK;
}

void dev_free(void* p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

}  // namespace qdb

using namespace qdb;

extern "C" {

const char* qdb_last_error(void) { return g_last_error.c_str(); }

int64_t qdb_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* qdb_version(void) { return "qikkdb_b200 0.1 (sm_100a)"; }

int32_t qdb_device_count(int32_t* out_count) {
    if (!out_count) return fail(QDB_ERR_INVALID, "qdb_device_count: null out_count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    *out_count = n;
    return QDB_OK;
}

int32_t qdb_malloc(void** out_ptr, int64_t bytes, void* stream) {
    if (!out_ptr || bytes < 0) return fail(QDB_ERR_INVALID, "qdb_malloc: bad arguments");
    return dev_alloc(out_ptr, static_cast<size_t>(bytes), as_stream(stream));
}

int32_t qdb_free(void* ptr, void* stream) {
    if (!ptr) return QDB_OK;
    QDB_CUDA_TRY(cudaFreeAsync(ptr, as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_memcpy_h2d(void* dst, const void* src, int64_t bytes, void* stream) {
    if (bytes <= 0) return QDB_OK;
    QDB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_memcpy_d2h(void* dst, const void* src, int64_t bytes, void* stream) {
    if (bytes <= 0) return QDB_OK;
    QDB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_memcpy_d2d(void* dst, const void* src, int64_t bytes, void* stream) {
    if (bytes <= 0) return QDB_OK;
    QDB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_memset(void* dst, int32_t byte_value, int64_t bytes, void* stream) {
    if (bytes <= 0) return QDB_OK;
    QDB_CUDA_TRY(cudaMemsetAsync(dst, byte_value, bytes, as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_stream_sync(void* stream) {
    QDB_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
    return QDB_OK;
}

int32_t qdb_set_device(int32_t device) {
    QDB_CUDA_TRY(cudaSetDevice(device));
    return QDB_OK;
}

int32_t qdb_get_device(int32_t* out_device) {
    if (!out_device) return fail(QDB_ERR_INVALID, "qdb_get_device: null out_device");
    int d = 0;
    QDB_CUDA_TRY(cudaGetDevice(&d));
    *out_device = d;
    return QDB_OK;
}

int32_t qdb_memcpy_peer(void* dst, int32_t dst_device, const void* src, int32_t src_device, int64_t bytes) {
    if (bytes <= 0) return QDB_OK;
    QDB_CUDA_TRY(cudaMemcpyPeer(dst, dst_device, src, src_device, static_cast<size_t>(bytes)));
    return QDB_OK;
}

}  // extern "C"
