// Dot product over the LEAF tiles that allocates no memory.
//
// Who needs it: a caller that may not enter the CUDA allocator at the point of the
// call.  One example is a simulator that reserved the GPU's memory for its own pool up
// front, where any further cudaMalloc can fail.  Another is a time-critical loop that
// must not call cudaFree: cudaFree synchronises the whole device and stalls work on
// every other stream.  cmg_amg_dot allocates its reduction scratch on first use per
// grid; this variant keeps its scratch in a fixed array in the module's global memory
// instead.
//
// Limits and rules:
//  * at most kNoAllocMaxLeafTiles LEAF tiles (one partial sum per tile); larger grids
//    are rejected with CMG_ERR_INVALID before anything is launched;
//  * each call clears the arrival counter (a scratch word) on its stream before its
//    launch (cudaMemsetAsync, which allocates nothing) and poisons the result word with a
//    NaN, so a call never depends on what an earlier call left in the array;
//  * the scratch is shared by all calls on a device, so calls that overlap in time
//    (other streams, other host threads) race on it and give wrong results -- the
//    overlapping calls only, since the next ordered call starts clean.  A call whose
//    result word still holds the NaN after its launch reports CMG_ERR_CUDA.  Calls must
//    be ordered, e.g. on one stream;
//  * the call runs on the grid's device (the one current when its device copy was
//    first allocated), switching to it and back if another device is current;
//  * the first call on each device looks up the array's device address for that device
//    (cudaGetSymbolAddress, with the device current); later calls reuse it.  Make one
//    call on each device before the time-critical part starts.  The cached address is
//    not refreshed after cudaDeviceReset, so do not use this entry point across one.
// The arithmetic and summation order are those of k_dot, so the result equals
// cmg_amg_dot's bit for bit.
#include <cstring>
#include <mutex>

#include "kernels.hpp"

namespace cmg {

namespace {

constexpr int kNoAllocMaxLeafTiles = 16384;  // 8.4 M leaf cells; scratch 128 KB

// words [0, max): per-block partial sums (double bit patterns); [max]: the result;
// [max + 1]: arrival counter, zero between calls
static __device__ __align__(256) unsigned long long g_dot_scratch[kNoAllocMaxLeafTiles + 2];

__device__ __forceinline__ double dot4_na(const float4& a, const float4& b) {  // four products summed in float
    float f = __fmul_rn(a.x, b.x);
    f = __fmaf_rn(a.y, b.y, f);
    f = __fmaf_rn(a.z, b.z, f);
    f = __fmaf_rn(a.w, b.w, f);
    return (double)f;
}

__global__ void __launch_bounds__(128) k_dot_noalloc(const int* leaf, const float* A, const float* B, unsigned long long* scratch) {
    __shared__ double red[4];
    __shared__ bool is_last;
    const int t = leaf[blockIdx.x];
    const size_t base = (size_t)t * kCells + 4 * threadIdx.x;
    const double bs = block_sum128(dot4_na(ld4(A + base), ld4(B + base)), red);
    if (threadIdx.x == 0) scratch[blockIdx.x] = (unsigned long long)__double_as_longlong(bs);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(&scratch[kNoAllocMaxLeafTiles + 1], 1ull) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    double s = 0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 128) s += __longlong_as_double((long long)__ldcg(scratch + i));
    const double d = block_sum128(s, red);
    if (threadIdx.x == 0) {
        scratch[kNoAllocMaxLeafTiles] = (unsigned long long)__double_as_longlong(d);
        scratch[kNoAllocMaxLeafTiles + 1] = 0ull;
    }
}

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
unsigned long long* g_addr[kMaxDevices] = {};

// device address of the scratch array on device dev, which must be current (looked up
// once per device)
cudaError_t scratch_address(int dev, unsigned long long** out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

}  // namespace

int dot_noalloc_max_leaf_tiles() { return kNoAllocMaxLeafTiles; }

namespace {
// the call proper, with the grid's device current
cudaError_t dot_noalloc_on(int device, const int* leaf, int nleaf, const float* A, const float* B, double* out_host,
                           cudaStream_t st) {
    unsigned long long* scratch = nullptr;
    cudaError_t e = scratch_address(device, &scratch);
    if (e != cudaSuccess) return e;
    // counter to zero, result word to a NaN (all bits set): neither allocates
    e = cudaMemsetAsync(scratch + kNoAllocMaxLeafTiles + 1, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch + kNoAllocMaxLeafTiles, 0xff, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    note_kernel_launch();
    k_dot_noalloc<<<nleaf, 128, 0, st>>>(leaf, A, B, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    unsigned long long bits = 0;
    e = cudaMemcpyAsync(&bits, scratch + kNoAllocMaxLeafTiles, sizeof(bits), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    if (bits == ~0ull) return cudaErrorLaunchFailure;  // no block finished last: an overlapping call
    std::memcpy(out_host, &bits, sizeof(double));
    return cudaSuccess;
}
}  // namespace

cudaError_t dot_noalloc(int device, const int* leaf, int nleaf, const float* A, const float* B, double* out_host,
                        cudaStream_t st) {
    if (nleaf <= 0) {
        *out_host = 0.0;
        return cudaSuccess;
    }
    if (nleaf > kNoAllocMaxLeafTiles) return cudaErrorInvalidValue;
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    if (device < 0) device = cur;
    if (device != cur && (e = cudaSetDevice(device)) != cudaSuccess) return e;
    e = dot_noalloc_on(device, leaf, nleaf, A, B, out_host, st);
    if (device != cur) {
        const cudaError_t e2 = cudaSetDevice(cur);
        if (e == cudaSuccess) e = e2;
    }
    return e;
}

}  // namespace cmg
