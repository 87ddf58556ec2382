// hsc_spmv_noalloc: y = H x straight from the one-triangle BCOO, allocating
// nothing.
//
// Some callers of the solver's matrix product cannot allocate device memory
// at the moment they need it: an engine that reserves all of its device memory
// up front through its own pool leaves the CUDA heap nothing to give, and a
// simulation loop that overlaps assembly and solves on several streams cannot
// afford the device-wide synchronisation that cudaFree (and often cudaMalloc)
// implies.  hsc_spmv needs a context whose analysis allocates the row-owner
// BSR plan; this variant needs no context and no allocation: it accumulates
// H x in a fixed scratch array that lives in this file for as long as the
// library is loaded (8 MiB per GPU that loads it), then copies it to y, so y
// may even alias x.
//
// Limits and sharing: at most kNoAllocMaxDofs (1,048,576) dofs; larger systems
// are rejected with HSC_ERR_INVALID before anything is launched.  Every call
// on a device uses the same array and leaves the last call's sums in it; each
// call clears the part it uses first.  Calls that overlap on the GPU (on
// different streams, or from different host threads without ordering) race on
// the array and give wrong results: order them on one stream.  The first call
// on a device looks up the array's device address (cudaGetSymbolAddress, with
// that device current) and caches it; make that first call before any stream
// capture begins.  Under lazy module loading (CUDA_MODULE_LOADING=LAZY, the
// default since CUDA 12.2) the module that holds the array is loaded, and the
// array created, by that first call too: "allocates nothing" holds from the
// second call on a device.  The sums use FP64 atomics, so the last bits may
// differ from hsc_spmv's fixed-order row sums.
//
// There is no analysis step to validate the triplets, so the product kernel
// checks every block index against nblock itself: a triplet with a row or
// column outside [0, nblock) is skipped (nothing is read or written for it)
// and raises a second file-scope flag, which the call reads back after the
// product and turns into HSC_ERR_INVALID.  Reading the flag waits for the
// stream, so the call returns with y complete.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/hsc_c_api.h"

namespace {

constexpr long long kNoAllocMaxDofs = 1 << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_acc[kNoAllocMaxDofs];
// triplets the last call skipped because a block index was out of range
static __device__ int g_noalloc_bad;

std::mutex g_mutex;
double* g_acc_ptr[kMaxDevices] = {};

__global__ void noalloc_zero_kernel(double* acc, long long n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) g_noalloc_bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        acc[i] = 0.0;
}

// one thread per stored triplet: its block and, off the diagonal, its transpose
__global__ void noalloc_spmv_kernel(const int* rows, const int* cols, const double* vals, long long nnzb,
                                    int nblock, const double* x, double* acc) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= nnzb) return;
    const int r = rows[t], c = cols[t];
    if ((unsigned)r >= (unsigned)nblock || (unsigned)c >= (unsigned)nblock) {
        atomicAdd(&g_noalloc_bad, 1);
        return;
    }
    const double* B = vals + 9 * t;  // column-major: B(i, j) = B[i + 3 j]
    const double xc0 = x[3 * (long long)c], xc1 = x[3 * (long long)c + 1], xc2 = x[3 * (long long)c + 2];
    for (int i = 0; i < 3; ++i)
        atomicAdd(acc + 3 * (long long)r + i, B[i] * xc0 + B[i + 3] * xc1 + B[i + 6] * xc2);
    if (r != c) {
        const double xr0 = x[3 * (long long)r], xr1 = x[3 * (long long)r + 1], xr2 = x[3 * (long long)r + 2];
        for (int j = 0; j < 3; ++j)
            atomicAdd(acc + 3 * (long long)c + j, B[3 * j] * xr0 + B[3 * j + 1] * xr1 + B[3 * j + 2] * xr2);
    }
}

__global__ void noalloc_copy_kernel(const double* acc, double* y, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = acc[i];
}

// device address of the scratch array on the current device (looked up once)
int scratch_address(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return HSC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_acc_ptr[dev]) {
        double* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_noalloc_acc) != cudaSuccess || !p) return HSC_ERR_CUDA;
        g_acc_ptr[dev] = p;
    }
    *out = g_acc_ptr[dev];
    return HSC_OK;
}

}  // namespace

extern "C" int hsc_spmv_noalloc(const hsc_bcoo3* A, const double* d_x, double* d_y, void* stream) {
    if (!A || !d_x || !d_y || A->nnzb < 0 || A->nblock <= 0) return HSC_ERR_INVALID;
    if ((A->nnzb > 0 && (!A->d_rows || !A->d_cols || !A->d_values))) return HSC_ERR_INVALID;
    const long long n = 3LL * A->nblock;
    if (n > kNoAllocMaxDofs) return HSC_ERR_INVALID;  // beyond the fixed scratch array
    // an error left pending by the caller's own earlier work is not ours to
    // report or to clear: refuse to launch behind it
    if (cudaPeekAtLastError() != cudaSuccess) return HSC_ERR_CUDA;
    double* acc = nullptr;
    const int rc = scratch_address(&acc);
    if (rc != HSC_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int grid_n = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    noalloc_zero_kernel<<<grid_n, 256, 0, st>>>(acc, n);
    if (cudaGetLastError() != cudaSuccess) return HSC_ERR_CUDA;
    if (A->nnzb > 0) {
        noalloc_spmv_kernel<<<(unsigned)((A->nnzb + 255) / 256), 256, 0, st>>>(A->d_rows, A->d_cols, A->d_values,
                                                                              A->nnzb, A->nblock, d_x, acc);
        if (cudaGetLastError() != cudaSuccess) return HSC_ERR_CUDA;
    }
    noalloc_copy_kernel<<<grid_n, 256, 0, st>>>(acc, d_y, n);
    if (cudaGetLastError() != cudaSuccess) return HSC_ERR_CUDA;
    int bad = 0;
    if (cudaMemcpyFromSymbolAsync(&bad, g_noalloc_bad, sizeof(int), 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return HSC_ERR_CUDA;
    return bad ? HSC_ERR_INVALID : HSC_OK;
}
